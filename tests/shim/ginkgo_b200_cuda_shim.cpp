// The maintainer-side shim that puts libginkgo_b200 behind Ginkgo's CUDA
// kernel interface: definitions of gko::kernels::cuda::<ns>::<kernel> (the
// functions the GKO_DECLARE_* macros declare and libginkgo_cuda normally
// provides) that call the C ABI of include/ginkgo_b200.h, and the
// solver-level hook of Cg.  tests/test_shim_compiles.py compiles this file
// against the reference's own headers, with the kernel declarations and
// instantiation macros of core/, so every signature here is checked against
// the reference; INTEGRATION.md quotes it.
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include <ginkgo/core/base/exception_helpers.hpp>
#include <ginkgo/core/base/executor.hpp>
#include <ginkgo/core/matrix/csr.hpp>
#include <ginkgo/core/matrix/dense.hpp>
#include <ginkgo/core/matrix/ell.hpp>
#include <ginkgo/core/matrix/sellp.hpp>
#include <ginkgo/core/preconditioner/jacobi.hpp>
#include <ginkgo/core/solver/cg.hpp>
#include <ginkgo/core/stop/combined.hpp>
#include <ginkgo/core/stop/iteration.hpp>
#include <ginkgo/core/stop/residual_norm.hpp>

#include "core/base/mixed_precision_types.hpp"
#include "core/matrix/csr_builder.hpp"
#include "core/matrix/csr_kernels.hpp"
#include "core/matrix/ell_kernels.hpp"
#include "core/matrix/sellp_kernels.hpp"
#include "ginkgo_b200.h"


// A negative status of the C ABI as Ginkgo's exceptions.
#define B2S_GKO_CALL(expr)                                                    \
    do {                                                                      \
        const int rc_ = (expr);                                               \
        if (rc_ == B2S_ERR_INVALID_ARG || rc_ == B2S_ERR_UNSUPPORTED) {       \
            throw ::gko::NotSupported(__FILE__, __LINE__, #expr,              \
                                      b2s_last_error());                      \
        }                                                                     \
        if (rc_ == B2S_ERR_CUDA) {                                            \
            throw ::gko::CudaError(__FILE__, __LINE__, #expr, 0);             \
        }                                                                     \
        if (rc_ < 0) throw ::gko::Error(__FILE__, __LINE__, b2s_last_error()); \
    } while (false)


namespace gko {
namespace b2s_shim {

template <typename T>
constexpr int value_code()
{
    return std::is_same_v<T, double> ? B2S_VALUE_F64
           : std::is_same_v<T, float> ? B2S_VALUE_F32
                                      : -1;
}

template <typename... T>
constexpr bool all_real_f32_f64 = ((value_code<T>() >= 0) && ...);

// The longest row, as the classical and automatical strategies record it;
// measured on the device for the other strategies.
template <typename V>
int64 max_row_nnz_of(std::shared_ptr<const CudaExecutor> exec, const matrix::Csr<V, int32>* a)
{
    using Csr = matrix::Csr<V, int32>;
    auto strat = a->get_strategy();
    if (auto c = std::dynamic_pointer_cast<typename Csr::classical>(strat)) {
        return c->get_max_length_per_row();
    }
    if (auto c = std::dynamic_pointer_cast<typename Csr::automatical>(strat)) {
        return c->get_max_length_per_row();
    }
    array<int64> ws(exec, 1);
    int64 out = 0;
    B2S_GKO_CALL(b2s_csr_max_row_nnz(a->get_size()[0], a->get_const_row_ptrs(), &out,
                                     ws.get_data(), exec->get_stream()));
    return out;
}

// The load_balance partition of a matrix (the role of srow), built once on
// the device and kept per matrix.
template <typename V>
const int32* tiles_of(std::shared_ptr<const CudaExecutor> exec,
                      const matrix::Csr<V, int32>* a, int64* num_tiles)
{
    static std::mutex m;
    static std::map<const void*, array<int32>> cache;
    const int64 n = a->get_size()[0];
    const int64 nnz = a->get_num_stored_elements();
    *num_tiles = b2s_csr_load_balance_num_tiles(n, nnz);
    std::lock_guard<std::mutex> lock(m);
    auto it = cache.find(a);
    if (it == cache.end() || it->second.get_size() != size_type(*num_tiles + 1)) {
        array<int32> tiles(exec, *num_tiles + 1);
        B2S_GKO_CALL(b2s_csr_load_balance_setup(n, nnz, a->get_const_row_ptrs(), *num_tiles,
                                                tiles.get_data(), exec->get_stream()));
        it = cache.insert_or_assign(a, std::move(tiles)).first;
    }
    return it->second.get_const_data();
}

}  // namespace b2s_shim


namespace kernels {
namespace cuda {
namespace csr {


template <typename MatrixValueType, typename InputValueType, typename OutputValueType,
          typename IndexType>
void advanced_spmv(std::shared_ptr<const DefaultExecutor> exec,
                   matrix::view::dense<const MatrixValueType> alpha,
                   const matrix::Csr<MatrixValueType, IndexType>* a,
                   matrix::view::dense<const InputValueType> b,
                   matrix::view::dense<const OutputValueType> beta,
                   matrix::view::dense<OutputValueType> c);


template <typename MatrixValueType, typename InputValueType, typename OutputValueType,
          typename IndexType>
void spmv(std::shared_ptr<const DefaultExecutor> exec,
          const matrix::Csr<MatrixValueType, IndexType>* a,
          matrix::view::dense<const InputValueType> b,
          matrix::view::dense<OutputValueType> c)
{
    if constexpr (!std::is_same_v<IndexType, int32> ||
                  !b2s_shim::all_real_f32_f64<MatrixValueType, InputValueType,
                                              OutputValueType>) {
        GKO_NOT_IMPLEMENTED;
    } else {
        const int64 n = a->get_size()[0], m = a->get_size()[1];
        const int64 mrn = b2s_shim::max_row_nnz_of(exec, a);
        if constexpr (std::is_same_v<MatrixValueType, InputValueType> &&
                      std::is_same_v<MatrixValueType, OutputValueType>) {
            const bool lb = a->get_strategy()->get_name() == "load_balance";
            int64 nt = 0;
            const int32* tiles = lb ? b2s_shim::tiles_of(exec, a, &nt) : nullptr;
            if constexpr (std::is_same_v<MatrixValueType, double>) {
                B2S_GKO_CALL(b2s_csr_spmv_f64(
                    lb ? B2S_CSR_LOAD_BALANCE : B2S_CSR_CLASSICAL, n, m,
                    a->get_const_row_ptrs(), a->get_const_col_idxs(), a->get_const_values(),
                    mrn, tiles, nt, b.values, b.stride, c.values, c.stride, c.size[1],
                    nullptr, nullptr, exec->get_stream()));
            } else {
                B2S_GKO_CALL(b2s_csr_spmv_f32(
                    lb ? B2S_CSR_LOAD_BALANCE : B2S_CSR_CLASSICAL, n, m,
                    a->get_const_row_ptrs(), a->get_const_col_idxs(), a->get_const_values(),
                    mrn, tiles, nt, b.values, b.stride, c.values, c.stride, c.size[1],
                    nullptr, nullptr, exec->get_stream()));
            }
        } else {
            // mixed value types: the most precise of the three
            B2S_GKO_CALL(b2s_csr_spmv_mixed(
                b2s_shim::value_code<MatrixValueType>(),
                b2s_shim::value_code<InputValueType>(),
                b2s_shim::value_code<OutputValueType>(), n, m, a->get_const_row_ptrs(),
                a->get_const_col_idxs(), a->get_const_values(), mrn, b.values, b.stride,
                c.values, c.stride, c.size[1], nullptr, nullptr, exec->get_stream()));
        }
    }
}

template <typename MatrixValueType, typename InputValueType, typename OutputValueType,
          typename IndexType>
void advanced_spmv(std::shared_ptr<const DefaultExecutor> exec,
                   matrix::view::dense<const MatrixValueType> alpha,
                   const matrix::Csr<MatrixValueType, IndexType>* a,
                   matrix::view::dense<const InputValueType> b,
                   matrix::view::dense<const OutputValueType> beta,
                   matrix::view::dense<OutputValueType> c)
{
    if constexpr (!std::is_same_v<IndexType, int32> ||
                  !b2s_shim::all_real_f32_f64<MatrixValueType, InputValueType,
                                              OutputValueType>) {
        GKO_NOT_IMPLEMENTED;
    } else {
        const int64 n = a->get_size()[0], m = a->get_size()[1];
        // alpha and beta are device scalars in the operand types
        B2S_GKO_CALL(b2s_csr_spmv_mixed(
            b2s_shim::value_code<MatrixValueType>(), b2s_shim::value_code<InputValueType>(),
            b2s_shim::value_code<OutputValueType>(), n, m, a->get_const_row_ptrs(),
            a->get_const_col_idxs(), a->get_const_values(),
            b2s_shim::max_row_nnz_of(exec, a), b.values, b.stride, c.values, c.stride,
            c.size[1], alpha.values, beta.values, exec->get_stream()));
    }
}

template <typename ValueType, typename IndexType>
void spgemm(std::shared_ptr<const DefaultExecutor> exec,
            const matrix::Csr<ValueType, IndexType>* a,
            const matrix::Csr<ValueType, IndexType>* b, matrix::Csr<ValueType, IndexType>* c)
{
    if constexpr (!std::is_same_v<IndexType, int32> ||
                  !b2s_shim::all_real_f32_f64<ValueType>) {
        GKO_NOT_IMPLEMENTED;
    } else {
        const int64 n = a->get_size()[0], m = b->get_size()[1];
        array<char> ws(exec, b2s_csr_spgemm_workspace_bytes(n, m));
        int64 nnz = 0;
        B2S_GKO_CALL(b2s_csr_spgemm_symbolic(
            n, m, a->get_const_row_ptrs(), a->get_const_col_idxs(), b->get_const_row_ptrs(),
            b->get_const_col_idxs(), nullptr, nullptr, c->get_row_ptrs(), &nnz,
            ws.get_data(), ws.get_size(), exec->get_stream()));
        matrix::CsrBuilder<ValueType, IndexType> builder{c};
        builder.get_col_idx_array().resize_and_reset(nnz);
        builder.get_value_array().resize_and_reset(nnz);
        if constexpr (std::is_same_v<ValueType, double>) {
            B2S_GKO_CALL(b2s_csr_spgemm_numeric_f64(
                n, m, nullptr, a->get_const_row_ptrs(), a->get_const_col_idxs(),
                a->get_const_values(), b->get_const_row_ptrs(), b->get_const_col_idxs(),
                b->get_const_values(), nullptr, nullptr, nullptr, nullptr,
                c->get_const_row_ptrs(), builder.get_col_idx_array().get_data(),
                builder.get_value_array().get_data(), ws.get_data(), ws.get_size(),
                exec->get_stream()));
        } else {
            B2S_GKO_CALL(b2s_csr_spgemm_numeric_f32(
                n, m, nullptr, a->get_const_row_ptrs(), a->get_const_col_idxs(),
                a->get_const_values(), b->get_const_row_ptrs(), b->get_const_col_idxs(),
                b->get_const_values(), nullptr, nullptr, nullptr, nullptr,
                c->get_const_row_ptrs(), builder.get_col_idx_array().get_data(),
                builder.get_value_array().get_data(), ws.get_data(), ws.get_size(),
                exec->get_stream()));
        }
    }
}

GKO_INSTANTIATE_FOR_EACH_MIXED_VALUE_AND_INDEX_TYPE(GKO_DECLARE_CSR_SPMV_KERNEL);
GKO_INSTANTIATE_FOR_EACH_MIXED_VALUE_AND_INDEX_TYPE(GKO_DECLARE_CSR_ADVANCED_SPMV_KERNEL);
GKO_INSTANTIATE_FOR_EACH_VALUE_AND_INDEX_TYPE(GKO_DECLARE_CSR_SPGEMM_KERNEL);


}  // namespace csr


namespace ell {


template <typename InputValueType, typename MatrixValueType, typename OutputValueType,
          typename IndexType>
void spmv(std::shared_ptr<const DefaultExecutor> exec,
          const matrix::Ell<MatrixValueType, IndexType>* a,
          matrix::view::dense<const InputValueType> b, matrix::view::dense<OutputValueType> c)
{
    if constexpr (!std::is_same_v<IndexType, int32> ||
                  !b2s_shim::all_real_f32_f64<MatrixValueType, InputValueType,
                                              OutputValueType>) {
        GKO_NOT_IMPLEMENTED;
    } else {
        B2S_GKO_CALL(b2s_ell_spmv_mixed(
            b2s_shim::value_code<MatrixValueType>(), b2s_shim::value_code<InputValueType>(),
            b2s_shim::value_code<OutputValueType>(), a->get_size()[0], a->get_size()[1],
            a->get_num_stored_elements_per_row(), a->get_stride(), a->get_const_col_idxs(),
            a->get_const_values(), b.values, b.stride, c.values, c.stride, c.size[1], nullptr,
            nullptr, exec->get_stream()));
    }
}

GKO_INSTANTIATE_FOR_EACH_MIXED_VALUE_AND_INDEX_TYPE(GKO_DECLARE_ELL_SPMV_KERNEL);


}  // namespace ell


namespace sellp {


template <typename IndexType>
void compute_slice_sets(std::shared_ptr<const DefaultExecutor> exec,
                        const array<IndexType>& row_ptrs, size_type slice_size,
                        size_type stride_factor, size_type* slice_sets,
                        size_type* slice_lengths)
{
    if constexpr (!std::is_same_v<IndexType, int32>) {
        GKO_NOT_IMPLEMENTED;
    } else {
        const int64 n = int64(row_ptrs.get_size()) - 1;
        array<char> ws(exec, b2s_sellp_slice_sets_workspace_bytes(n, slice_size));
        B2S_GKO_CALL(b2s_sellp_compute_slice_sets(
            n, row_ptrs.get_const_data(), slice_size, stride_factor,
            reinterpret_cast<uint64_t*>(slice_sets), reinterpret_cast<uint64_t*>(slice_lengths),
            ws.get_data(), ws.get_size(), exec->get_stream()));
    }
}

GKO_INSTANTIATE_FOR_EACH_INDEX_TYPE(GKO_DECLARE_SELLP_COMPUTE_SLICE_SETS_KERNEL);


}  // namespace sellp
}  // namespace cuda
}  // namespace kernels


namespace b2s_shim {

// (max_iters, reduction_factor, residual_mode) of a criterion factory that
// the fused solvers support: Iteration plus at most one ResidualNorm or
// ImplicitResidualNorm, alone or inside a Combined; false for anything else.
template <typename V>
bool criteria_of(const stop::CriterionFactory* f, int64* max_iters, double* reduction,
                 int* mode)
{
    auto base = [](stop::mode b) {
        return b == stop::mode::initial_resnorm ? B2S_BASELINE_INITIAL_RESNORM
               : b == stop::mode::absolute      ? B2S_BASELINE_ABSOLUTE
                                                : B2S_BASELINE_RHS_NORM;
    };
    if (auto it = dynamic_cast<const stop::Iteration::Factory*>(f)) {
        *max_iters = std::min<int64>(*max_iters, it->get_parameters().max_iters);
        return true;
    }
    if (auto r = dynamic_cast<const typename stop::ResidualNorm<V>::Factory*>(f)) {
        *reduction = r->get_parameters().reduction_factor;
        *mode = base(r->get_parameters().baseline);
        return true;
    }
    if (auto r = dynamic_cast<const typename stop::ImplicitResidualNorm<V>::Factory*>(f)) {
        *reduction = r->get_parameters().reduction_factor;
        *mode = base(r->get_parameters().baseline) | B2S_STOP_IMPLICIT;
        return true;
    }
    if (auto c = dynamic_cast<const stop::Combined::Factory*>(f)) {
        for (const auto& sub : c->get_parameters().criteria) {
            if (!criteria_of<V>(sub.get(), max_iters, reduction, mode)) return false;
        }
        return true;
    }
    return false;
}

// The inverted diagonal of a scalar Jacobi preconditioner (max_block_size 1:
// the interleaved block storage is then the plain inverse diagonal), null
// for no preconditioner; false for any other preconditioner.
template <typename V>
bool scalar_jacobi_of(const LinOp* p, const V** inv_diag)
{
    *inv_diag = nullptr;
    if (p == nullptr || dynamic_cast<const matrix::Identity<V>*>(p)) return true;
    if (auto j = dynamic_cast<const preconditioner::Jacobi<V, int32>*>(p)) {
        if (j->get_parameters().max_block_size != 1) return false;
        *inv_diag = j->get_blocks();
        return true;
    }
    return false;
}

// A block Jacobi preconditioner in full precision (max_block_size > 1, no
// storage optimisation): its blocks are already in the interleaved layout
// the fused solvers read, delimited by the first num_blocks + 1 entries of
// the block_pointers parameter that generate() filled in.
template <typename V>
bool block_jacobi_of(const LinOp* p, int64* num_blocks, const int32** ptrs,
                     int* max_block_size, const V** blocks)
{
    auto j = dynamic_cast<const preconditioner::Jacobi<V, int32>*>(p);
    if (j == nullptr) return false;
    const auto& par = j->get_parameters();
    const auto& opt = par.storage_optimization;
    if (par.max_block_size <= 1 || opt.is_block_wise ||
        precision_reduction::storage_type(opt.of_all_blocks) != 0) {
        return false;
    }
    *num_blocks = static_cast<int64>(j->get_num_blocks());
    *ptrs = par.block_pointers.get_const_data();
    *max_block_size = static_cast<int>(par.max_block_size);
    *blocks = j->get_blocks();
    return true;
}

// The solver-level hook of Cg<double>::apply_dense_impl on a CudaExecutor:
// the whole loop in one fused call.  Returns false (nothing done) when the
// combination is not the fused path's, so the caller runs the stock loop.
inline bool try_cg(const solver::Cg<double>* solver, const matrix::Dense<double>* b,
                   matrix::Dense<double>* x)
{
    auto exec = std::dynamic_pointer_cast<const CudaExecutor>(solver->get_executor());
    auto csr = std::dynamic_pointer_cast<const matrix::Csr<double, int32>>(
        solver->get_system_matrix());
    if (!exec || !csr || b->get_size()[1] > 16) return false;
    const double* inv_diag = nullptr;
    int64 num_blocks = 0;
    const int32* block_ptrs = nullptr;
    int max_block_size = 0;
    const double* blocks = nullptr;
    const LinOp* prec = solver->get_preconditioner().get();
    const bool block = block_jacobi_of<double>(prec, &num_blocks, &block_ptrs, &max_block_size,
                                               &blocks);
    if (!block && !scalar_jacobi_of<double>(prec, &inv_diag)) return false;
    int64 max_iters = std::numeric_limits<int64>::max();
    double reduction = 0.0;
    int mode = B2S_BASELINE_RHS_NORM;
    if (!criteria_of<double>(solver->get_stop_criterion_factory().get(), &max_iters,
                             &reduction, &mode)) {
        return false;
    }
    const int64 n = csr->get_size()[0], k = b->get_size()[1];
    int64 iters = 0;
    std::vector<double> res(k);
    std::vector<uint8_t> status(k);  // gko::stopping_status bit layout
    if (block) {
        array<char> ws(exec, b2s_cg_block_workspace_bytes(n, k, sizeof(double)));
        B2S_GKO_CALL(b2s_cg_block_solve_f64(
            n, csr->get_const_row_ptrs(), csr->get_const_col_idxs(), csr->get_const_values(),
            max_row_nnz_of(exec, csr.get()), num_blocks, block_ptrs, max_block_size,
            /*block_precisions=*/nullptr, blocks,
            b->get_const_values(), b->get_stride(), x->get_values(), x->get_stride(), k,
            max_iters, reduction, mode, /*check_every=*/8, ws.get_data(), ws.get_size(),
            &iters, res.data(), status.data(), exec->get_stream()));
        return true;
    }
    array<char> ws(exec, b2s_cg_workspace_bytes(n, k, sizeof(double)));
    B2S_GKO_CALL(b2s_cg_solve_f64(
        n, csr->get_const_row_ptrs(), csr->get_const_col_idxs(), csr->get_const_values(),
        max_row_nnz_of(exec, csr.get()), inv_diag, b->get_const_values(), b->get_stride(),
        x->get_values(), x->get_stride(), k, max_iters, reduction, mode,
        /*check_every=*/8, ws.get_data(), ws.get_size(), &iters, res.data(), status.data(),
        exec->get_stream()));
    return true;
}

}  // namespace b2s_shim
}  // namespace gko
