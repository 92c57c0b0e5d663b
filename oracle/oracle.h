/*
 * CPU oracle for the sparse iterative-solve path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the Ginkgo 1.12 ReferenceExecutor kernels and of
 * the executor-agnostic solver loops in core/solver/*.cpp.  It is the checker
 * for the CUDA library (tests, smoke check, the CPU baseline leg of the
 * benchmark) and is never linked into, loaded by or called from the product
 * library.  Every function cites the reference file:line it follows.
 *
 * Pinning: the reference cannot be compiled from a few source files (it needs
 * its own CMake build and a CMake-generated ginkgo/config.hpp), so the oracle
 * is pinned against the known-answer values in the reference's own tests
 * (reference/test/**), transcribed into tests/golden/known_answers.json.
 *
 * Conventions (reference include/ginkgo/core/matrix/device_views.hpp:24-43):
 * dense blocks are row-major n x k with a leading dimension (stride) `ld`.
 * Index type is int32, Sellp slice pointers are uint64 (size_type).
 * Functions exist for double (_f64) and float (_f32) value types; every
 * float kernel accumulates in float, as highest_precision<float,...> does.
 */
#ifndef GINKGO_B200_ORACLE_H
#define GINKGO_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_DECL(T, S)                                                        \
    void orc_csr_spmv_##S(int64_t n, const int32_t* rp, const int32_t* ci,    \
                          const T* v, const T* x, int64_t ldx, T* y,          \
                          int64_t ldy, int64_t k, const T* alpha,             \
                          const T* beta);                                     \
    void orc_csr_spmv_par_##S(int64_t n, const int32_t* rp,                   \
                              const int32_t* ci, const T* v, const T* x,      \
                              int64_t ldx, T* y, int64_t ldy, int64_t k,      \
                              int nthreads);                                  \
    void orc_ell_spmv_##S(int64_t n, int64_t width, int64_t stride,           \
                          const int32_t* ci, const T* v, const T* x,          \
                          int64_t ldx, T* y, int64_t ldy, int64_t k,          \
                          const T* alpha, const T* beta);                     \
    void orc_sellp_spmv_##S(int64_t n, int64_t slice_size,                    \
                            const uint64_t* slice_sets,                       \
                            const uint64_t* slice_lengths,                    \
                            const int32_t* ci, const T* v, const T* x,        \
                            int64_t ldx, T* y, int64_t ldy, int64_t k,        \
                            const T* alpha, const T* beta);                   \
    void orc_csr_to_ell_##S(int64_t n, const int32_t* rp, const int32_t* ci,  \
                            const T* v, int64_t width, int64_t stride,        \
                            int32_t* ell_ci, T* ell_v);                       \
    void orc_csr_to_sellp_##S(int64_t n, const int32_t* rp,                   \
                              const int32_t* ci, const T* v,                  \
                              int64_t slice_size, const uint64_t* slice_sets, \
                              const uint64_t* slice_lengths, int32_t* s_ci,   \
                              T* s_v);                                        \
    void orc_csr_transpose_##S(int64_t nrows, int64_t ncols,                  \
                               const int32_t* rp, const int32_t* ci,          \
                               const T* v, int32_t* t_rp, int32_t* t_ci,      \
                               T* t_v);                                       \
    void orc_jacobi_invert_diagonal_##S(int64_t n, const int32_t* rp,         \
                                        const int32_t* ci, const T* v,        \
                                        T* inv_diag);                         \
    void orc_cg_step_1_##S(int64_t n, int64_t k, T* p, const T* z,           \
                           const T* rho, const T* prev_rho,                   \
                           const char* stopped);                              \
    void orc_cg_step_2_##S(int64_t n, int64_t k, T* x, T* r, const T* p,      \
                           const T* q, const T* beta, const T* rho,           \
                           const char* stopped);                              \
    void orc_gmres_hessenberg_qr_##S(int64_t k, int64_t iter, T* givens_sin,  \
                                     T* givens_cos, T* residual_norm, T* rnc, \
                                     T* hessenberg_iter,                      \
                                     int64_t* final_iter_nums,                \
                                     const char* stopped);                    \
    void orc_gmres_solve_krylov_##S(int64_t k, const T* rnc,                  \
                                    const T* hessenberg, int64_t ld_h, T* y,  \
                                    const int64_t* final_iter_nums,           \
                                    const char* finalized);                   \
    int orc_cg_##S(int64_t n, const int32_t* rp, const int32_t* ci,           \
                   const T* v, const T* inv_diag, const T* b, T* x,           \
                   int64_t k, int max_iters, double reduction, int mode,      \
                   int* iters_out, double* res_norm_out);                     \
    int orc_cg_block_##S(int64_t n, const int32_t* rp, const int32_t* ci,     \
                         const T* v, int64_t nblocks, const int32_t* bptrs,   \
                         int max_bs, const T* binv, const T* b, T* x,         \
                         int64_t k, int max_iters, double reduction,          \
                         int mode, int* iters_out, double* res_norm_out);                     \
    int orc_bicgstab_##S(int64_t n, const int32_t* rp, const int32_t* ci,     \
                         const T* v, const T* inv_diag, const T* b, T* x,     \
                         int max_iters, double reduction, int mode,           \
                         int* iters_out, double* res_norm_out);               \
    int orc_bicgstab_block_##S(int64_t n, const int32_t* rp,                  \
                               const int32_t* ci, const T* v, int64_t nblocks,\
                               const int32_t* bptrs, int max_bs,              \
                               const T* binv, const T* b, T* x,               \
                               int max_iters, double reduction, int mode,     \
                               int* iters_out, double* res_norm_out);               \
    int orc_gmres_##S(int64_t n, const int32_t* rp, const int32_t* ci,        \
                      const T* v, const T* inv_diag, const T* b, T* x,        \
                      int krylov_dim, int ortho, int max_iters,               \
                      double reduction, int mode, int* iters_out,             \
                      double* res_norm_out);                                  \
    int orc_gmres_block_##S(int64_t n, const int32_t* rp, const int32_t* ci,  \
                            const T* v, int64_t nblocks, const int32_t* bptrs,\
                            int max_bs, const T* binv, const T* b, T* x,      \
                            int krylov_dim, int ortho, int max_iters,         \
                            double reduction, int mode, int* iters_out,       \
                            double* res_norm_out);                                  \
    int orc_batch_bicgstab_ell_##S(int64_t n, int64_t width, int64_t stride,  \
                                   const int32_t* ci, const T* v,             \
                                   const T* b, T* x, int max_iters,           \
                                   double tol, int use_jacobi,                \
                                   int* iters_out, double* res_norm_out);

ORC_DECL(double, f64)
ORC_DECL(float, f32)
#undef ORC_DECL

/* Sellp slice layout (reference/matrix/sellp_kernels.cpp:109-131). */
void orc_sellp_compute_slice_sets(int64_t n, const int32_t* rp,
                                  int64_t slice_size, int64_t stride_factor,
                                  uint64_t* slice_sets,
                                  uint64_t* slice_lengths);
/* Ell width (common/unified/matrix/ell_kernels.cpp:26-40). */
int64_t orc_csr_max_row_nnz(int64_t n, const int32_t* rp);

/* Iterative refinement with an FP64 outer residual and an FP32 GMRES inner
 * solve (core/solver/ir.cpp:191-257 with a Gmres<float> inner solver, as in
 * examples/mixed-precision-ir/mixed-precision-ir.cpp). */
int orc_ir_gmres_mixed(int64_t n, const int32_t* rp, const int32_t* ci,
                       const double* v, const double* b, double* x,
                       int krylov_dim, int inner_iters, double inner_reduction,
                       int max_outer, double reduction, int* outer_out,
                       int* inner_total_out, double* res_norm_out);

#ifdef __cplusplus
}
#endif

#endif
