/*
 * libginkgo_b200 — C ABI of the B200 (sm_100a) sparse iterative-solve path.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*, the cudaStream_t value; NULL = legacy default stream),
 * launches asynchronously on that stream unless documented otherwise, and
 * returns B2S_OK (0) or a negative B2S_ERR_* code; b2s_last_error() then
 * holds a message.  The library allocates no device memory: where scratch
 * space is needed the caller passes a workspace of the size the matching
 * *_workspace_bytes() query reports, as the reference's kernels take a
 * gko::array<char> from the executor.
 *
 * Data layout (the reference's):
 *   Csr    row_ptrs int32[n+1], col_idxs int32[nnz], values[nnz]
 *          (include/ginkgo/core/matrix/csr.hpp)
 *   Ell    column-major, entry i of row r at r + i*stride, padding column -1
 *          (include/ginkgo/core/matrix/ell.hpp:31-41)
 *   Sellp  entry i of local row l in slice s at (slice_sets[s] + i)*slice_size
 *          + l; slice_sets/slice_lengths are uint64 (size_type)
 *          (include/ginkgo/core/matrix/sellp.hpp:379-383)
 *   Dense  row-major n x k with leading dimension ld (matrix::view::dense,
 *          include/ginkgo/core/matrix/device_views.hpp:24-43)
 * Scalars alpha/beta are device pointers to one value (a 1x1 Dense); both
 * NULL selects the simple form c = A b.  beta == 0 ignores c (NaN included).
 *
 * Each declaration names the reference kernel interface it stands in for.
 */
#ifndef GINKGO_B200_H
#define GINKGO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2S_VERSION 1

#define B2S_OK 0
#define B2S_ERR_INVALID_ARG -1
#define B2S_ERR_CUDA -2
#define B2S_ERR_WORKSPACE -3
#define B2S_ERR_UNSUPPORTED -4

#define B2S_CSR_CLASSICAL 0
#define B2S_CSR_LOAD_BALANCE 1

/* Message of the last failed call on this host thread. */
const char* b2s_last_error(void);
/* B2S_VERSION of the loaded library. */
int b2s_version(void);

/* ---------------------------------------------------------------- SpMV -- */

/* Size of the load_balance partition: the stored entries are cut into
 * nc = ceil(nnz / 256) chunks of consecutive entries (at least one), each
 * SpMV warp sums the rows whose last entry lies in its chunk and leaves a
 * partial sum for a row that continues past it.  The partition array has
 * num_tiles + 1 = 34 nc + 4 int32 entries (8-byte aligned): the first row of
 * every chunk, the continuing row of every chunk and the partial-sum
 * scratch every SpMV rewrites (SpMVs of one matrix must not overlap on the
 * GPU).  Stands in for the host computed srow of Csr::load_balance
 * (include/ginkgo/core/matrix/csr.hpp:417-468, make_srow :1651-1655). */
int64_t b2s_csr_load_balance_num_tiles(int64_t num_rows, int64_t nnz);
/* Builds the load_balance partition on the GPU (one binary search per
 * chunk); called once per matrix like Csr::make_srow. */
int b2s_csr_load_balance_setup(int64_t num_rows, int64_t nnz,
                               const int32_t* row_ptrs, int64_t num_tiles,
                               int32_t* tile_rows, void* stream);

/* c = A b or c = alpha A b + beta c for Csr A.
 * strategy B2S_CSR_CLASSICAL: subwarp per row sized from max_row_nnz;
 * strategy B2S_CSR_LOAD_BALANCE: tile_rows/num_tiles from the setup above.
 * Replaces csr::spmv / csr::advanced_spmv
 * (core/matrix/csr_kernels.hpp:29-42; CUDA dispatch
 * common/cuda_hip/matrix/csr_kernels.template.cpp:2368-2485). */
int b2s_csr_spmv_f64(int strategy, int64_t num_rows, int64_t num_cols,
                     const int32_t* row_ptrs, const int32_t* col_idxs,
                     const double* values, int64_t max_row_nnz,
                     const int32_t* tile_rows, int64_t num_tiles,
                     const double* b, int64_t ldb, double* c, int64_t ldc,
                     int64_t num_rhs, const double* alpha, const double* beta,
                     void* stream);
int b2s_csr_spmv_f32(int strategy, int64_t num_rows, int64_t num_cols,
                     const int32_t* row_ptrs, const int32_t* col_idxs,
                     const float* values, int64_t max_row_nnz,
                     const int32_t* tile_rows, int64_t num_tiles,
                     const float* b, int64_t ldb, float* c, int64_t ldc,
                     int64_t num_rhs, const float* alpha, const float* beta,
                     void* stream);

/* Ell SpMV; replaces ell::spmv / ell::advanced_spmv
 * (core/matrix/ell_kernels.hpp:21-35). */
int b2s_ell_spmv_f64(int64_t num_rows, int64_t num_cols, int64_t width,
                     int64_t stride, const int32_t* col_idxs,
                     const double* values, const double* b, int64_t ldb,
                     double* c, int64_t ldc, int64_t num_rhs,
                     const double* alpha, const double* beta, void* stream);
int b2s_ell_spmv_f32(int64_t num_rows, int64_t num_cols, int64_t width,
                     int64_t stride, const int32_t* col_idxs,
                     const float* values, const float* b, int64_t ldb,
                     float* c, int64_t ldc, int64_t num_rhs,
                     const float* alpha, const float* beta, void* stream);

/* Sellp SpMV; replaces sellp::spmv / sellp::advanced_spmv
 * (core/matrix/sellp_kernels.hpp:21-35). */
int b2s_sellp_spmv_f64(int64_t num_rows, int64_t num_cols, int64_t slice_size,
                       const uint64_t* slice_sets,
                       const uint64_t* slice_lengths, const int32_t* col_idxs,
                       const double* values, const double* b, int64_t ldb,
                       double* c, int64_t ldc, int64_t num_rhs,
                       const double* alpha, const double* beta, void* stream);
int b2s_sellp_spmv_f32(int64_t num_rows, int64_t num_cols, int64_t slice_size,
                       const uint64_t* slice_sets,
                       const uint64_t* slice_lengths, const int32_t* col_idxs,
                       const float* values, const float* b, int64_t ldb,
                       float* c, int64_t ldc, int64_t num_rhs,
                       const float* alpha, const float* beta, void* stream);
/* The same with the caller's knowledge of the longest slice
 * (max_slice_length = the largest slice_lengths entry; 0 when not known):
 * with four or more right-hand sides, slices of at most 64 entries per row
 * let each lane slot take two neighbouring rows. */
int b2s_sellp_spmv_hinted_f64(int64_t num_rows, int64_t num_cols, int64_t slice_size,
                              const uint64_t* slice_sets, const uint64_t* slice_lengths,
                              const int32_t* col_idxs, const double* values, const double* b,
                              int64_t ldb, double* c, int64_t ldc, int64_t num_rhs,
                              const double* alpha, const double* beta,
                              int64_t max_slice_length, void* stream);
int b2s_sellp_spmv_hinted_f32(int64_t num_rows, int64_t num_cols, int64_t slice_size,
                              const uint64_t* slice_sets, const uint64_t* slice_lengths,
                              const int32_t* col_idxs, const float* values, const float* b,
                              int64_t ldb, float* c, int64_t ldc, int64_t num_rhs,
                              const float* alpha, const float* beta,
                              int64_t max_slice_length, void* stream);

/* Value type codes of the mixed-type entry points. */
#define B2S_VALUE_F64 0
#define B2S_VALUE_F32 1

/* Csr and Ell SpMV with the matrix, b and c each FP64 or FP32 (type codes
 * B2S_VALUE_*), computed in the most precise of the three; replaces the
 * mixed instantiations of csr::spmv / csr::advanced_spmv and ell::spmv /
 * ell::advanced_spmv (GKO_INSTANTIATE_FOR_EACH_MIXED_VALUE_AND_INDEX_TYPE,
 * core/matrix/csr_kernels.hpp:29-42, core/matrix/ell_kernels.hpp:21-26;
 * highest_precision arithmetic as in common/cuda_hip/matrix/
 * csr_kernels.template.cpp:2109-2110).  alpha has the matrix type and beta
 * the output type (core/matrix/csr.cpp:301-311); both or neither.  Csr rows
 * are summed by a subwarp sized from max_row_nnz (any strategy); uniform
 * types are accepted, but b2s_csr_spmv_f64/_f32 and b2s_ell_spmv_* are
 * their tuned path. */
int b2s_csr_spmv_mixed(int matrix_type, int input_type, int output_type,
                       int64_t num_rows, int64_t num_cols, const int32_t* row_ptrs,
                       const int32_t* col_idxs, const void* values,
                       int64_t max_row_nnz, const void* b, int64_t ldb, void* c,
                       int64_t ldc, int64_t num_rhs, const void* alpha,
                       const void* beta, void* stream);
int b2s_ell_spmv_mixed(int matrix_type, int input_type, int output_type,
                       int64_t num_rows, int64_t num_cols, int64_t width, int64_t stride,
                       const int32_t* col_idxs, const void* values, const void* b,
                       int64_t ldb, void* c, int64_t ldc, int64_t num_rhs,
                       const void* alpha, const void* beta, void* stream);

/* dst = src converted between FP64 and FP32 (num_rows x num_cols,
 * row-major with leading dimensions): the temporary conversions of
 * make_temporary_conversion (include/ginkgo/core/base/
 * precision_dispatch.hpp:43-83) for operands whose type differs from the
 * operator's, e.g. Sellp, which computes in its own type only
 * (core/matrix/sellp.cpp:150-180). */
int b2s_dense_convert(int src_type, int dst_type, int64_t num_rows, int64_t num_cols,
                      const void* src, int64_t lds, void* dst, int64_t ldd, void* stream);

/* ------------------------------------------------------- conversions -- */

/* Longest row; synchronises the stream and writes *result on the host.
 * workspace: 8 device bytes.  Replaces ell::compute_max_row_nnz
 * (core/matrix/ell_kernels.hpp:37-40). */
int b2s_csr_max_row_nnz(int64_t num_rows, const int32_t* row_ptrs,
                        int64_t* result, void* workspace, void* stream);

/* Csr -> Ell with the given width and stride (>= num_rows); replaces
 * csr::convert_to_ell (core/matrix/csr_kernels.hpp:99-103). */
int b2s_csr_convert_to_ell_f64(int64_t num_rows, const int32_t* row_ptrs,
                               const int32_t* col_idxs, const double* values,
                               int64_t width, int64_t stride,
                               int32_t* ell_col_idxs, double* ell_values,
                               void* stream);
int b2s_csr_convert_to_ell_f32(int64_t num_rows, const int32_t* row_ptrs,
                               const int32_t* col_idxs, const float* values,
                               int64_t width, int64_t stride,
                               int32_t* ell_col_idxs, float* ell_values,
                               void* stream);

/* Sellp slice lengths (max row length per slice rounded up to
 * stride_factor) and slice_sets (num_slices + 1 entries, exclusive prefix
 * sum); replaces sellp::compute_slice_sets
 * (core/matrix/sellp_kernels.hpp:41-45). */
int64_t b2s_sellp_slice_sets_workspace_bytes(int64_t num_rows,
                                             int64_t slice_size);
int b2s_sellp_compute_slice_sets(int64_t num_rows, const int32_t* row_ptrs,
                                 int64_t slice_size, int64_t stride_factor,
                                 uint64_t* slice_sets, uint64_t* slice_lengths,
                                 void* workspace, int64_t workspace_bytes,
                                 void* stream);

/* The same slice lengths and slice sets as b2s_sellp_compute_slice_sets,
 * for callers that cannot allocate device memory: a host that gives this
 * library one fixed device arena and forbids further allocations, or a
 * latency-sensitive loop that must not call cudaMalloc because it can
 * synchronise the whole device.  It takes no workspace: its scan scratch is
 * a 32 KiB array inside the library (4096 uint64 entries), so it handles at
 * most 8,386,560 slices per call and rejects more with B2S_ERR_INVALID_ARG.
 * The first call on a device looks up the array's device address once (with
 * that device current); make that first call before any stream capture.
 * The address is kept for the life of the process and is not looked up
 * again after cudaDeviceReset or a reset of the primary context: do not
 * call this entry point on a device after resetting it.
 * All calls share the array, so calls that overlap on the GPU race.  It
 * allocates nothing.  No counterpart in the reference: Ginkgo always takes
 * its scratch from the executor. */
int b2s_sellp_compute_slice_sets_noalloc(int64_t num_rows,
                                         const int32_t* row_ptrs,
                                         int64_t slice_size,
                                         int64_t stride_factor,
                                         uint64_t* slice_sets,
                                         uint64_t* slice_lengths,
                                         void* stream);

/* Csr -> Sellp scatter into slice_sets[num_slices] * slice_size slots;
 * replaces csr::convert_to_sellp (core/matrix/csr_kernels.hpp:117-120). */
int b2s_csr_convert_to_sellp_f64(int64_t num_rows, const int32_t* row_ptrs,
                                 const int32_t* col_idxs, const double* values,
                                 int64_t slice_size, const uint64_t* slice_sets,
                                 const uint64_t* slice_lengths,
                                 int32_t* sellp_col_idxs, double* sellp_values,
                                 void* stream);
int b2s_csr_convert_to_sellp_f32(int64_t num_rows, const int32_t* row_ptrs,
                                 const int32_t* col_idxs, const float* values,
                                 int64_t slice_size, const uint64_t* slice_sets,
                                 const uint64_t* slice_lengths,
                                 int32_t* sellp_col_idxs, float* sellp_values,
                                 void* stream);

/* Transpose (num_cols x num_rows result, columns sorted, same order as the
 * reference's sequential scatter); replaces csr::transpose
 * (core/matrix/csr_kernels.hpp:122-125; cuSPARSE csr2csc in
 * common/cuda_hip/matrix/csr_kernels.template.cpp:3010-3056). */
int64_t b2s_csr_transpose_workspace_bytes(int64_t num_rows, int64_t num_cols,
                                          int64_t nnz, int value_bytes);
int b2s_csr_transpose_f64(int64_t num_rows, int64_t num_cols, int64_t nnz,
                          const int32_t* row_ptrs, const int32_t* col_idxs,
                          const double* values, int32_t* t_row_ptrs,
                          int32_t* t_col_idxs, double* t_values,
                          void* workspace, int64_t workspace_bytes,
                          void* stream);
int b2s_csr_transpose_f32(int64_t num_rows, int64_t num_cols, int64_t nnz,
                          const int32_t* row_ptrs, const int32_t* col_idxs,
                          const float* values, int32_t* t_row_ptrs,
                          int32_t* t_col_idxs, float* t_values,
                          void* workspace, int64_t workspace_bytes,
                          void* stream);

/* --------------------------------------------------------- Jacobi ------ */

/* inv_diag = 1 / diag(A), 1 where the diagonal is zero or missing;
 * aggregate_l1 != 0 first adds the absolute sum of each row's off-diagonal
 * entries to its diagonal (Jacobi's aggregate_l1, scalar_l1).  Replaces the
 * scalar Jacobi generate (jacobi::invert_diagonal,
 * core/preconditioner/jacobi_kernels.hpp:42-45, after extract_diagonal and
 * scalar_l1, core/preconditioner/jacobi.cpp:337-369). */
int b2s_jacobi_invert_diagonal_f64(int64_t num_rows, const int32_t* row_ptrs,
                                   const int32_t* col_idxs,
                                   const double* values, double* inv_diag,
                                   int aggregate_l1, void* stream);
int b2s_jacobi_invert_diagonal_f32(int64_t num_rows, const int32_t* row_ptrs,
                                   const int32_t* col_idxs,
                                   const float* values, float* inv_diag,
                                   int aggregate_l1, void* stream);
/* x = inv_diag .* b, or alpha inv_diag .* b + beta x; replaces
 * jacobi::simple_scalar_apply / scalar_apply
 * (core/preconditioner/jacobi_kernels.hpp:61-65, 79-85). */
int b2s_jacobi_apply_f64(int64_t num_rows, int64_t num_rhs,
                         const double* inv_diag, const double* b, int64_t ldb,
                         double* x, int64_t ldx, const double* alpha,
                         const double* beta, void* stream);
int b2s_jacobi_apply_f32(int64_t num_rows, int64_t num_rhs,
                         const float* inv_diag, const float* b, int64_t ldb,
                         float* x, int64_t ldx, const float* alpha,
                         const float* beta, void* stream);

/* Block Jacobi with full-precision blocks of at most max_block_size <= 32
 * rows.  block_ptrs (device, num_blocks + 1 entries, from 0 to num_rows)
 * delimit the diagonal blocks; a block with a bad extent is skipped.  The
 * inverses use the reference's block-interleaved layout
 * (block_interleaved_storage_scheme, include/ginkgo/core/preconditioner/
 * jacobi.hpp:37-140, with the CUDA block stride of 32): with
 * gs = 32 / pow2ceil(max_block_size) blocks per group, entry (i, j) of
 * block b is at (b >> group_power) * group_offset + (b % gs) * block_offset
 * + i + j * stride, stride = gs * max_block_size; b2s_jacobi_storage_scheme
 * gives block_offset, group_offset, group_power and the storage space (in
 * values) for num_blocks blocks, the values Jacobi::get_storage_scheme()
 * and the blocks array of the reference hold.  Generate: Gauss-Jordan with partial pivoting
 * in place (the first row of largest magnitude is the pivot; a zero pivot
 * ends the elimination of that block, as the reference's invert_block
 * does); replaces jacobi::generate (core/preconditioner/jacobi_kernels.hpp,
 * reference/preconditioner/jacobi_kernels.cpp:310-395) without adaptive
 * precision.  Apply: x = D^-1 b or alpha D^-1 b + beta x (beta == 0 ignores
 * x); replaces jacobi::simple_apply / apply. */
/* Block pointers for block Jacobi, computed on the host from HOST arrays:
 * runs of consecutive rows with identical column patterns, cut at
 * max_block_size rows (natural blocks), then neighbouring natural blocks
 * merged while the sum stays within max_block_size; jacobi::find_blocks
 * (reference/preconditioner/jacobi_kernels.cpp:28-98).  block_ptrs_out
 * holds num_rows + 1 entries; returns the number of blocks, or a negative
 * B2S_ERR_* code. */
int64_t b2s_jacobi_find_blocks(int64_t num_rows, const int32_t* row_ptrs,
                               const int32_t* col_idxs, int max_block_size,
                               int32_t* block_ptrs_out);
int b2s_jacobi_storage_scheme(int max_block_size, int64_t num_blocks, int64_t* block_offset,
                              int64_t* group_offset, int32_t* group_power,
                              int64_t* storage_space);
/* aggregate_l1 != 0: each row's diagonal entry first gains the absolute sum
 * of the row's entries outside its block (block_l1, reference/
 * preconditioner/jacobi_kernels.cpp:751-779, a missing diagonal counting as
 * 0 as after add_diagonal_elements). */
int b2s_jacobi_block_generate_f64(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const double* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, double* blocks, int aggregate_l1,
                                  void* stream);
int b2s_jacobi_block_generate_f32(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const float* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, float* blocks, int aggregate_l1,
                                  void* stream);
int b2s_jacobi_block_apply_f64(int64_t num_rows, int64_t num_blocks,
                               const int32_t* block_ptrs, int max_block_size,
                               const double* blocks, const double* b, int64_t ldb,
                               double* x, int64_t ldx, int64_t num_rhs,
                               const double* alpha, const double* beta, void* stream);
int b2s_jacobi_block_apply_f32(int64_t num_rows, int64_t num_blocks,
                               const int32_t* block_ptrs, int max_block_size,
                               const float* blocks, const float* b, int64_t ldb,
                               float* x, int64_t ldx, int64_t num_rhs,
                               const float* alpha, const float* beta, void* stream);

/* Adaptive-precision block Jacobi (Jacobi's storage_optimization; replaces
 * jacobi::generate / apply / simple_apply with block_precisions,
 * reference/preconditioner/jacobi_kernels.cpp:309-450, and the CUDA
 * executor's adaptive instantiations of the same kernels).  Precisions are
 * precision_reduction bytes, (preserving << 4) | non-preserving: 0x00 full,
 * 0x01 reduce, 0x02 reduce twice, 0x10 truncate, 0x11 truncate the reduced
 * type, 0x20 truncate twice, 0xff autodetect.  The blocks of one group
 * (32 / pow2ceil(max_block_size) blocks) share the most reduced precision all
 * of them support; a reduced group stores its values as an array of the
 * storage type (FP32, FP16, or the top 32 / 16 bits of the value) with the
 * interleaved indexing, from the start of the group's slot.
 *
 * generate_adaptive: block_precisions (num_blocks bytes, device) holds the
 * requested precision of each block on entry and the chosen one on return;
 * conditioning (num_blocks values) receives ||B||_inf ||B^-1||_inf per
 * block; accuracy bounds cond * eps of an accepted storage; workspace holds
 * b2s_jacobi_adaptive_workspace_bytes bytes.  apply_adaptive is
 * b2s_jacobi_block_apply_* reading each group at its precision.
 * expand widens the reduced storage to full precision (same layout, values
 * exact) into full_blocks, reduce rounds full-precision storage to the
 * given precisions; both work in place as well. */
int b2s_jacobi_adaptive_workspace_bytes(int64_t num_blocks, int64_t* bytes);
int b2s_jacobi_block_generate_adaptive_f64(int64_t num_rows, const int32_t* row_ptrs,
                                           const int32_t* col_idxs, const double* values,
                                           int64_t num_blocks, const int32_t* block_ptrs,
                                           int max_block_size, double accuracy,
                                           double* conditioning, uint8_t* block_precisions,
                                           double* blocks, int aggregate_l1, void* workspace,
                                           void* stream);
int b2s_jacobi_block_generate_adaptive_f32(int64_t num_rows, const int32_t* row_ptrs,
                                           const int32_t* col_idxs, const float* values,
                                           int64_t num_blocks, const int32_t* block_ptrs,
                                           int max_block_size, float accuracy,
                                           float* conditioning, uint8_t* block_precisions,
                                           float* blocks, int aggregate_l1, void* workspace,
                                           void* stream);
int b2s_jacobi_block_apply_adaptive_f64(int64_t num_rows, int64_t num_blocks,
                                        const int32_t* block_ptrs, int max_block_size,
                                        const uint8_t* block_precisions, const double* blocks,
                                        const double* b, int64_t ldb, double* x, int64_t ldx,
                                        int64_t num_rhs, const double* alpha,
                                        const double* beta, void* stream);
int b2s_jacobi_block_apply_adaptive_f32(int64_t num_rows, int64_t num_blocks,
                                        const int32_t* block_ptrs, int max_block_size,
                                        const uint8_t* block_precisions, const float* blocks,
                                        const float* b, int64_t ldb, float* x, int64_t ldx,
                                        int64_t num_rhs, const float* alpha,
                                        const float* beta, void* stream);
int b2s_jacobi_block_expand_f64(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const double* blocks,
                                double* full_blocks, void* stream);
int b2s_jacobi_block_expand_f32(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const float* blocks,
                                float* full_blocks, void* stream);
int b2s_jacobi_block_reduce_f64(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const double* full_blocks,
                                double* blocks, void* stream);
int b2s_jacobi_block_reduce_f32(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const float* full_blocks,
                                float* blocks, void* stream);

/* ------------------------------------------------ Krylov step kernels -- */

/* Kernel-level stand-ins for a caller that keeps the reference's solver
 * loop.  Dense operands are row-major (values, stride); scalars are device
 * arrays of k = num_rhs entries; stop_status is the reference's
 * stopping_status array (one uint8 per column: bit 7 converged, bit 6
 * finalized, bits 0-5 criterion id). */

/* cg::initialize / step_1 / step_2 (core/solver/cg_kernels.hpp:25-52). */
int b2s_cg_initialize_f64(int64_t n, int64_t k, const double* b, int64_t ldb,
                          double* r, int64_t ldr, double* z, int64_t ldz,
                          double* p, int64_t ldp, double* q, int64_t ldq,
                          double* prev_rho, double* rho, uint8_t* stop_status,
                          void* stream);
int b2s_cg_initialize_f32(int64_t n, int64_t k, const float* b, int64_t ldb,
                          float* r, int64_t ldr, float* z, int64_t ldz,
                          float* p, int64_t ldp, float* q, int64_t ldq,
                          float* prev_rho, float* rho, uint8_t* stop_status,
                          void* stream);
int b2s_cg_step_1_f64(int64_t n, int64_t k, double* p, int64_t ldp,
                      const double* z, int64_t ldz, const double* rho,
                      const double* prev_rho, const uint8_t* stop_status,
                      void* stream);
int b2s_cg_step_1_f32(int64_t n, int64_t k, float* p, int64_t ldp,
                      const float* z, int64_t ldz, const float* rho,
                      const float* prev_rho, const uint8_t* stop_status,
                      void* stream);
int b2s_cg_step_2_f64(int64_t n, int64_t k, double* x, int64_t ldx, double* r,
                      int64_t ldr, const double* p, int64_t ldp,
                      const double* q, int64_t ldq, const double* beta,
                      const double* rho, const uint8_t* stop_status,
                      void* stream);
int b2s_cg_step_2_f32(int64_t n, int64_t k, float* x, int64_t ldx, float* r,
                      int64_t ldr, const float* p, int64_t ldp, const float* q,
                      int64_t ldq, const float* beta, const float* rho,
                      const uint8_t* stop_status, void* stream);

/* bicgstab::step_1 / step_2 / step_3 / finalize
 * (core/solver/bicgstab_kernels.hpp:42-88). */
int b2s_bicgstab_step_1_f64(int64_t n, int64_t k, const double* r,
                            int64_t ldr, double* p, int64_t ldp,
                            const double* v, int64_t ldv, const double* rho,
                            const double* prev_rho, const double* alpha,
                            const double* omega, const uint8_t* stop_status,
                            void* stream);
int b2s_bicgstab_step_1_f32(int64_t n, int64_t k, const float* r, int64_t ldr,
                            float* p, int64_t ldp, const float* v, int64_t ldv,
                            const float* rho, const float* prev_rho,
                            const float* alpha, const float* omega,
                            const uint8_t* stop_status, void* stream);
int b2s_bicgstab_step_2_f64(int64_t n, int64_t k, const double* r,
                            int64_t ldr, double* s, int64_t lds,
                            const double* v, int64_t ldv, const double* rho,
                            double* alpha, const double* beta,
                            const uint8_t* stop_status, void* stream);
int b2s_bicgstab_step_2_f32(int64_t n, int64_t k, const float* r, int64_t ldr,
                            float* s, int64_t lds, const float* v, int64_t ldv,
                            const float* rho, float* alpha, const float* beta,
                            const uint8_t* stop_status, void* stream);
int b2s_bicgstab_step_3_f64(int64_t n, int64_t k, double* x, int64_t ldx,
                            double* r, int64_t ldr, const double* s,
                            int64_t lds, const double* t, int64_t ldt,
                            const double* y, int64_t ldy, const double* z,
                            int64_t ldz, const double* alpha,
                            const double* beta, const double* gamma,
                            double* omega, const uint8_t* stop_status,
                            void* stream);
int b2s_bicgstab_step_3_f32(int64_t n, int64_t k, float* x, int64_t ldx,
                            float* r, int64_t ldr, const float* s, int64_t lds,
                            const float* t, int64_t ldt, const float* y,
                            int64_t ldy, const float* z, int64_t ldz,
                            const float* alpha, const float* beta,
                            const float* gamma, float* omega,
                            const uint8_t* stop_status, void* stream);
int b2s_bicgstab_finalize_f64(int64_t n, int64_t k, double* x, int64_t ldx,
                              const double* y, int64_t ldy,
                              const double* alpha, uint8_t* stop_status,
                              void* stream);
int b2s_bicgstab_finalize_f32(int64_t n, int64_t k, float* x, int64_t ldx,
                              const float* y, int64_t ldy, const float* alpha,
                              uint8_t* stop_status, void* stream);

/* common_gmres::hessenberg_qr and solve_krylov
 * (core/solver/common_gmres_kernels.hpp:32-50): hessenberg_iter is
 * (iter + 2) x k, givens_* krylov_dim x k, residual_norm_collection
 * (krylov_dim + 1) x k; hessenberg(j, i * k + c) holds H(i, j). */
int b2s_gmres_hessenberg_qr_f64(int64_t k, int64_t iter, double* givens_sin,
                                int64_t ld_sin, double* givens_cos,
                                int64_t ld_cos, double* residual_norm,
                                double* residual_norm_collection,
                                int64_t ld_rnc, double* hessenberg_iter,
                                int64_t ld_h, int64_t* final_iter_nums,
                                const uint8_t* stop_status, void* stream);
int b2s_gmres_hessenberg_qr_f32(int64_t k, int64_t iter, float* givens_sin,
                                int64_t ld_sin, float* givens_cos,
                                int64_t ld_cos, float* residual_norm,
                                float* residual_norm_collection,
                                int64_t ld_rnc, float* hessenberg_iter,
                                int64_t ld_h, int64_t* final_iter_nums,
                                const uint8_t* stop_status, void* stream);
int b2s_gmres_solve_krylov_f64(int64_t k,
                               const double* residual_norm_collection,
                               int64_t ld_rnc, const double* hessenberg,
                               int64_t ld_h, double* y, int64_t ld_y,
                               const int64_t* final_iter_nums,
                               const uint8_t* stop_status, void* stream);
int b2s_gmres_solve_krylov_f32(int64_t k, const float* residual_norm_collection,
                               int64_t ld_rnc, const float* hessenberg,
                               int64_t ld_h, float* y, int64_t ld_y,
                               const int64_t* final_iter_nums,
                               const uint8_t* stop_status, void* stream);

/* dense::compute_conj_dot / compute_norm2 per column, result on the device
 * (core/matrix/dense_kernels.hpp:100-118); deterministic two-level sum.
 * workspace: b2s_dense_reduction_workspace_bytes(k, value_bytes). */
int64_t b2s_dense_reduction_workspace_bytes(int64_t num_rhs, int value_bytes);
int b2s_dense_compute_dot_f64(int64_t n, int64_t k, const double* a,
                              int64_t lda, const double* b, int64_t ldb,
                              double* result, void* workspace,
                              int64_t workspace_bytes, void* stream);
int b2s_dense_compute_dot_f32(int64_t n, int64_t k, const float* a,
                              int64_t lda, const float* b, int64_t ldb,
                              float* result, void* workspace,
                              int64_t workspace_bytes, void* stream);
int b2s_dense_compute_norm2_f64(int64_t n, int64_t k, const double* a,
                                int64_t lda, double* result, void* workspace,
                                int64_t workspace_bytes, void* stream);
int b2s_dense_compute_norm2_f32(int64_t n, int64_t k, const float* a,
                                int64_t lda, float* result, void* workspace,
                                int64_t workspace_bytes, void* stream);

/* residual_norm::residual_norm (core/stop/residual_norm_kernels.hpp:21-29):
 * converges column c when tau[c] <= goal * orig_tau[c]; device_flags[0] is
 * cleared when an unstopped column is not converged (all converged),
 * device_flags[1] set when one changed.  The host reads the two flags. */
int b2s_residual_norm_check_f64(int64_t k, const double* tau,
                                const double* orig_tau, double goal,
                                int stopping_id, int set_finalized,
                                uint8_t* stop_status, int* device_flags,
                                void* stream);
int b2s_residual_norm_check_f32(int64_t k, const float* tau,
                                const float* orig_tau, double goal,
                                int stopping_id, int set_finalized,
                                uint8_t* stop_status, int* device_flags,
                                void* stream);

/* ------------------------------------------------------ fused solvers -- */

/* Whole-solve entry points.  They run the reference's solver loop on the
 * device with fused kernels and no host synchronisation inside an
 * iteration; the host checks the device stop flag once per replay of a
 * captured CUDA graph.  They synchronise `stream` before returning and
 * write the host outputs (iterations, residual norms, status).  Stopping:
 * Iteration(max_iters) + a residual criterion per right-hand-side column,
 * ||r|| <= reduction_factor * baseline, chosen by residual_mode (below);
 * status[j] uses the bit layout of
 * gko::stopping_status (include/ginkgo/core/stop/stopping_status.hpp):
 * bit 7 converged, bit 6 finalized, bits 0-5 criterion id (1 iteration
 * limit, 2 residual norm).  inv_diag: scalar Jacobi (from
 * b2s_jacobi_invert_diagonal_*) or NULL for no preconditioner. */

/* residual_mode of the fused solvers: the baseline of the residual goal
 * (stop::ResidualNorm's mode, include/ginkgo/core/stop/residual_norm.hpp:37:
 * rhs_norm ||b||, initial_resnorm ||b - A x_0||, absolute 1), with
 * B2S_STOP_IMPLICIT or-ed in for stop::ImplicitResidualNorm (:175), which
 * compares sqrt|rho| of the solver's implicit squared residual norm instead
 * of ||r|| (rho = r^T z for CG, r_hat^T r for BiCGStab: core/solver/cg.cpp:156,
 * core/solver/bicgstab.cpp:173).  GMRES takes a baseline only (the
 * reference's GMRES provides no implicit squared norm). */
#define B2S_BASELINE_RHS_NORM 0
#define B2S_BASELINE_INITIAL_RESNORM 1
#define B2S_BASELINE_ABSOLUTE 2
#define B2S_STOP_IMPLICIT 4

/* Preconditioned CG, 1..16 right-hand sides (b, x row-major with leading
 * dimensions).  Replaces Cg<V>::apply_dense_impl (core/solver/cg.cpp:91-189)
 * with cg::initialize/step_1/step_2 (core/solver/cg_kernels.hpp:25-52), the
 * dots, the Jacobi apply and residual_norm::residual_norm
 * (core/stop/residual_norm_kernels.hpp:21-29). */
int64_t b2s_cg_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                               int value_bytes);
int b2s_cg_solve_f64(int64_t num_rows, const int32_t* row_ptrs,
                     const int32_t* col_idxs, const double* values,
                     int64_t max_row_nnz, const double* inv_diag,
                     const double* b, int64_t ldb, double* x, int64_t ldx,
                     int64_t num_rhs, int64_t max_iters,
                     double reduction_factor, int residual_mode,
                     int64_t check_every,
                     void* workspace, int64_t workspace_bytes,
                     int64_t* iterations, double* residual_norms,
                     uint8_t* status, void* stream);
int b2s_cg_solve_f32(int64_t num_rows, const int32_t* row_ptrs,
                     const int32_t* col_idxs, const float* values,
                     int64_t max_row_nnz, const float* inv_diag,
                     const float* b, int64_t ldb, float* x, int64_t ldx,
                     int64_t num_rhs, int64_t max_iters,
                     double reduction_factor, int residual_mode,
                     int64_t check_every,
                     void* workspace, int64_t workspace_bytes,
                     int64_t* iterations, double* residual_norms,
                     uint8_t* status, void* stream);
/* CG preconditioned by block Jacobi: num_blocks blocks delimited by
 * block_ptrs (num_blocks + 1 entries covering 0..num_rows, each block at
 * most max_block_size rows), inverses in the interleaved storage that
 * b2s_jacobi_block_generate_* writes, or the adaptive storage of
 * b2s_jacobi_block_generate_adaptive_* with its block_precisions (NULL for
 * full-precision blocks; each group is read at its precision and widened).
 * z = M^-1 r is formed inside the update pass, one warp per group of
 * blocks, and stored; otherwise as
 * b2s_cg_solve_*.  The workspace query adds the stored z.  Replaces
 * Cg<V>::apply_dense_impl with a Jacobi<V> preconditioner of block size
 * > 1 (z = M r at core/solver/cg.cpp:146-149; Jacobi::apply_impl,
 * core/preconditioner/jacobi.cpp:150-168, simple_apply). */
int64_t b2s_cg_block_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                     int value_bytes);
int b2s_cg_block_solve_f64(int64_t num_rows, const int32_t* row_ptrs,
                           const int32_t* col_idxs, const double* values,
                           int64_t max_row_nnz, int64_t num_blocks,
                           const int32_t* block_ptrs, int max_block_size,
                           const uint8_t* block_precisions,
                           const double* blocks, const double* b, int64_t ldb,
                           double* x, int64_t ldx, int64_t num_rhs,
                           int64_t max_iters, double reduction_factor,
                           int residual_mode, int64_t check_every,
                           void* workspace, int64_t workspace_bytes,
                           int64_t* iterations, double* residual_norms,
                           uint8_t* status, void* stream);
int b2s_cg_block_solve_f32(int64_t num_rows, const int32_t* row_ptrs,
                           const int32_t* col_idxs, const float* values,
                           int64_t max_row_nnz, int64_t num_blocks,
                           const int32_t* block_ptrs, int max_block_size,
                           const uint8_t* block_precisions,
                           const float* blocks, const float* b, int64_t ldb,
                           float* x, int64_t ldx, int64_t num_rhs,
                           int64_t max_iters, double reduction_factor,
                           int residual_mode, int64_t check_every,
                           void* workspace, int64_t workspace_bytes,
                           int64_t* iterations, double* residual_norms,
                           uint8_t* status, void* stream);

/* Preconditioned BiCGStab, 1..16 right-hand sides.  Replaces
 * Bicgstab<V>::apply_dense_impl (core/solver/bicgstab.cpp:95-250) with
 * bicgstab::initialize/step_1/step_2/step_3/finalize
 * (core/solver/bicgstab_kernels.hpp:25-88). */
int64_t b2s_bicgstab_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                     int value_bytes);
int b2s_bicgstab_solve_f64(int64_t num_rows, const int32_t* row_ptrs,
                           const int32_t* col_idxs, const double* values,
                           int64_t max_row_nnz, const double* inv_diag,
                           const double* b, int64_t ldb, double* x,
                           int64_t ldx, int64_t num_rhs, int64_t max_iters,
                           double reduction_factor, int residual_mode,
                           int64_t check_every,
                           void* workspace, int64_t workspace_bytes,
                           int64_t* iterations, double* residual_norms,
                           uint8_t* status, void* stream);
int b2s_bicgstab_solve_f32(int64_t num_rows, const int32_t* row_ptrs,
                           const int32_t* col_idxs, const float* values,
                           int64_t max_row_nnz, const float* inv_diag,
                           const float* b, int64_t ldb, float* x, int64_t ldx,
                           int64_t num_rhs, int64_t max_iters,
                           double reduction_factor, int residual_mode,
                           int64_t check_every,
                           void* workspace, int64_t workspace_bytes,
                           int64_t* iterations, double* residual_norms,
                           uint8_t* status, void* stream);
/* BiCGStab preconditioned by block Jacobi (blocks as for
 * b2s_cg_block_solve_*): every iteration runs split, M p' and M s formed
 * one warp per block group right after p' and s and stored for the SpMVs
 * and the solution update; otherwise as b2s_bicgstab_solve_*.  The
 * workspace query adds the two stored vectors.  Replaces
 * Bicgstab<V>::apply_dense_impl with a Jacobi<V> of block size > 1
 * (preconditioner applies at core/solver/bicgstab.cpp:194 and :229). */
int64_t b2s_bicgstab_block_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                           int value_bytes);
int b2s_bicgstab_block_solve_f64(int64_t num_rows, const int32_t* row_ptrs,
                                 const int32_t* col_idxs, const double* values,
                                 int64_t max_row_nnz, int64_t num_blocks,
                                 const int32_t* block_ptrs, int max_block_size,
                                 const uint8_t* block_precisions,
                                 const double* blocks, const double* b, int64_t ldb,
                                 double* x, int64_t ldx, int64_t num_rhs,
                                 int64_t max_iters, double reduction_factor,
                                 int residual_mode, int64_t check_every,
                                 void* workspace, int64_t workspace_bytes,
                                 int64_t* iterations, double* residual_norms,
                                 uint8_t* status, void* stream);
int b2s_bicgstab_block_solve_f32(int64_t num_rows, const int32_t* row_ptrs,
                                 const int32_t* col_idxs, const float* values,
                                 int64_t max_row_nnz, int64_t num_blocks,
                                 const int32_t* block_ptrs, int max_block_size,
                                 const uint8_t* block_precisions,
                                 const float* blocks, const float* b, int64_t ldb,
                                 float* x, int64_t ldx, int64_t num_rhs,
                                 int64_t max_iters, double reduction_factor,
                                 int residual_mode, int64_t check_every,
                                 void* workspace, int64_t workspace_bytes,
                                 int64_t* iterations, double* residual_norms,
                                 uint8_t* status, void* stream);

#define B2S_GMRES_F64 0
#define B2S_GMRES_MIXED_F32 1
#define B2S_GMRES_MIXED_BF16 2
#define B2S_GMRES_CB_F32 3
#define B2S_GMRES_CB_F16 4
#define B2S_GMRES_CB_I64 5
#define B2S_GMRES_CB_I32 6
#define B2S_GMRES_CB_I16 7

/* Orthogonalisation of GMRES (solver::gmres::ortho_method,
 * include/ginkgo/core/solver/gmres.hpp:38-50).  CGS projects once
 * (h = V^T w); CGS2 projects twice, the second projection taken from the
 * Gram matrix of the basis in the same pass over it.  MGS, the reference's
 * default, runs as CGS2: one pass over the basis per Arnoldi step instead of
 * j + 1, with orthogonality at least as good; results agree with MGS to
 * rounding, iteration counts to within a few. */
#define B2S_ORTHO_MGS 0
#define B2S_ORTHO_CGS 1
#define B2S_ORTHO_CGS2 2

/* Restarted GMRES(krylov_dim), 1 <= krylov_dim <= 128 (larger values are
 * rejected with B2S_ERR_INVALID_ARG), right scalar-Jacobi preconditioning,
 * FP64 matrix/b/x/inv_diag; b and x are row-major num_rows x num_rhs with
 * leading dimensions ldb, ldx.  The columns are independent GMRES solves
 * (each with its own basis, Hessenberg matrix and stop status), run one
 * after the other.  variant B2S_GMRES_F64 is plain FP64 GMRES (Gmres<double>,
 * core/solver/gmres.cpp:325-640); B2S_GMRES_MIXED_F32 / _BF16 is iterative
 * refinement (Ir<double>, core/solver/ir.cpp:191-257) whose every outer step
 * computes r = b - A x and ||r|| in FP64 and runs one GMRES cycle on an FP32
 * copy of A with FP32 vectors and an FP32 or BF16 Krylov basis.  Hessenberg,
 * Givens and the triangular solve are FP64 in all variants.
 * B2S_GMRES_CB_F32 is compressed-basis GMRES (CbGmres<double> with
 * storage_precision reduce1, core/solver/cb_gmres.cpp): FP64 matrix, vectors
 * and arithmetic, the Krylov basis stored in FP32 and read back for the
 * orthogonalisation and the solution update.  B2S_GMRES_CB_F16, _I64,
 * _I32 and _I16 are CbGmres<double> with storage_precision reduce2, integer,
 * ireduce1 and ireduce2: the basis stored as the normalised vector in half,
 * or as trunc(v / s) in a 64-, 32- or 16-bit integer with one scale
 * s = (max|v| / ||v||) * 2 / INT_MAX per vector (core/solver/
 * cb_gmres_accessor.hpp); each new vector is formed in FP64 and then written
 * by a second pass once its norm and largest entry are known.  The
 * orthogonalisation of every CB-GMRES variant is the engine's CGS2 (the
 * reference re-orthogonalises CGS only while the norm drops below
 * 1/sqrt(2) of the previous one).  max_iters bounds the total
 * Arnoldi steps of a column; the goal is ||b - A x|| <= reduction_factor *
 * baseline on the explicit FP64 residual, baseline one of B2S_BASELINE_*
 * (||b||, the initial residual norm, or 1); inner_reduction ends an inner
 * cycle early once its estimate falls below inner_reduction * ||r||.  Per
 * column: iterations, restarts (cycles), residual_norms and status (the
 * reference's stopping_status bits: 0x80 converged, 0x40 finalized, low six
 * bits the criterion, 1 iteration limit, 2 residual norm); each output
 * array may be NULL.  max_row_nnz must be at least the longest row (the
 * workspace holds a column-major copy of A in the Arnoldi type when its
 * padding stays within a quarter of nnz; a longer row makes the solve
 * return B2S_ERR_INVALID_ARG). */
int64_t b2s_gmres_workspace_bytes(int64_t num_rows, int64_t nnz,
                                  int64_t max_row_nnz, int64_t num_rhs,
                                  int64_t krylov_dim, int variant);
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
                    uint8_t* status, void* stream);
/* GMRES (every variant above) right-preconditioned by block Jacobi:
 * num_blocks FP64 blocks delimited by block_ptrs (covering 0..num_rows, at
 * most max_block_size rows each), inverses in the interleaved storage of
 * b2s_jacobi_block_generate_f64.  Each SpMV input y = M V_j is formed in
 * place after the pass that writes V_j, one warp per block group, and the
 * cycle's update x += M V y likewise; an FP32 Arnoldi cycle rounds M y to
 * FP32.  Workspace as b2s_gmres_workspace_bytes.  Replaces the
 * preconditioner applies of Gmres<V>::apply_dense_impl with a Jacobi<V> of
 * block size > 1 (core/solver/gmres.cpp:530-531 on each Krylov vector,
 * :642-643 before the solution update). */
int b2s_gmres_block_solve(int variant, int ortho_method, int64_t num_rows,
                          const int32_t* row_ptrs, const int32_t* col_idxs,
                          const double* values, int64_t max_row_nnz,
                          int64_t num_blocks, const int32_t* block_ptrs,
                          int max_block_size, const uint8_t* block_precisions,
                          const double* blocks, const double* b, int64_t ldb,
                          double* x, int64_t ldx,
                          int64_t num_rhs, int64_t krylov_dim, int64_t max_iters,
                          double reduction_factor, int baseline,
                          double inner_reduction, void* workspace,
                          int64_t workspace_bytes, int64_t* iterations,
                          int64_t* restarts, double* residual_norms,
                          uint8_t* status, void* stream);

/* -------------------------------------------------------- gradients -- */

/* out[e] = alpha * sum_k u(row_e, k) * w(col_e, k) over the stored entries
 * of a Csr pattern (1..16 columns).  The backward of the differentiable
 * solve: with u = lambda, w = x, alpha = -1 it is dL/dA = -lambda x^T on A's
 * pattern.  No counterpart in the reference (it has no autograd path). */
int b2s_csr_sddmm_f64(int64_t num_rows, const int32_t* row_ptrs,
                      const int32_t* col_idxs, int64_t max_row_nnz,
                      const double* u, int64_t ldu, const double* w,
                      int64_t ldw, int64_t num_rhs, double alpha, double* out,
                      void* stream);
int b2s_csr_sddmm_f32(int64_t num_rows, const int32_t* row_ptrs,
                      const int32_t* col_idxs, int64_t max_row_nnz,
                      const float* u, int64_t ldu, const float* w,
                      int64_t ldw, int64_t num_rhs, double alpha, float* out,
                      void* stream);

/* ---------------------------------------------------- batched solver -- */

/* Batched BiCGStab over num_systems independent systems of uneven size in a
 * ragged batch Ell: system s has row_offsets[s+1] - row_offsets[s] rows
 * (1..2048) and its entries at values[width * row_offsets[s] + j * n_s + r]
 * (column-major per system, local column indices, -1 padding).  For equal
 * sizes this is the value layout of gko::batch::matrix::Ell
 * (include/ginkgo/core/matrix/batch_ell.hpp:149-221), column indices
 * stored per system.  b, x: concatenated per-system vectors (x = initial
 * guess in, solution out).  Stop: ||r|| <= tolerance * ||b|| (relative) or
 * ||r|| <= tolerance (tolerance_absolute != 0), or max_iters.  Outputs per
 * system on the device: iteration count and final residual norm (what
 * gko::batch::log::BatchConvergence records).  host_row_offsets: the same
 * offsets in host memory (used to sort systems into size buckets).
 * tune_table: NULL for the built-in choice, or 24 int32 from
 * b2s_batch_ell_bicgstab_tune_* (per size bucket 2^k rows: threads per
 * system, 1 = vectors in shared memory / 0 = global scratch).  Synchronises
 * the stream.  Replaces batch_bicgstab::apply
 * (core/solver/batch_bicgstab_kernels.hpp:177-190;
 * cuda/solver/batch_bicgstab_kernels.cu:24-153). */
int64_t b2s_batch_bicgstab_workspace_bytes(int64_t num_systems,
                                           int64_t total_rows,
                                           int value_bytes);
int b2s_batch_ell_bicgstab_solve_f64(
    int64_t num_systems, const int32_t* row_offsets,
    const int32_t* host_row_offsets, int64_t width, const int32_t* col_idxs,
    const double* values, const double* b, double* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    const int32_t* tune_table, void* workspace, int64_t workspace_bytes,
    int32_t* iterations, double* residual_norms, void* stream);
int b2s_batch_ell_bicgstab_solve_f32(
    int64_t num_systems, const int32_t* row_offsets,
    const int32_t* host_row_offsets, int64_t width, const int32_t* col_idxs,
    const float* values, const float* b, float* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    const int32_t* tune_table, void* workspace, int64_t workspace_bytes,
    int32_t* iterations, double* residual_norms, void* stream);
/* Autotuner: for every size bucket, times each threads-per-system and
 * vector-placement candidate on that bucket's systems (x restored between
 * trials), writes the fastest into tune_table_out (24 int32), then solves
 * with it. */
int b2s_batch_ell_bicgstab_tune_f64(
    int64_t num_systems, const int32_t* row_offsets,
    const int32_t* host_row_offsets, int64_t width, const int32_t* col_idxs,
    const double* values, const double* b, double* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    void* workspace, int64_t workspace_bytes, int32_t* iterations,
    double* residual_norms, int32_t* tune_table_out, void* stream);
int b2s_batch_ell_bicgstab_tune_f32(
    int64_t num_systems, const int32_t* row_offsets,
    const int32_t* host_row_offsets, int64_t width, const int32_t* col_idxs,
    const float* values, const float* b, float* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    void* workspace, int64_t workspace_bytes, int32_t* iterations,
    double* residual_norms, int32_t* tune_table_out, void* stream);

/* The same solve on the reference's uniform batch::matrix::Ell
 * (include/ginkgo/core/matrix/batch_ell.hpp:149-221, core/matrix/
 * batch_struct.hpp:268-280): num_systems systems of num_rows rows
 * (1..2048), one col_idxs array of num_rows * width entries shared by all
 * systems, values[s * num_rows * width + j * num_rows + r].  With
 * tune_table_out non-NULL the call autotunes (and solves) as
 * b2s_batch_ell_bicgstab_tune_*; otherwise tune_table (or NULL) selects the
 * configuration.  Workspace as b2s_batch_bicgstab_workspace_bytes with
 * total_rows = num_systems * num_rows. */
int b2s_batch_ell_uniform_bicgstab_solve_f64(
    int64_t num_systems, int64_t num_rows, int64_t width, const int32_t* col_idxs,
    const double* values, const double* b, double* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    const int32_t* tune_table, void* workspace, int64_t workspace_bytes,
    int32_t* iterations, double* residual_norms, void* stream, int32_t* tune_table_out);
int b2s_batch_ell_uniform_bicgstab_solve_f32(
    int64_t num_systems, int64_t num_rows, int64_t width, const int32_t* col_idxs,
    const float* values, const float* b, float* x, int64_t max_iters,
    double tolerance, int tolerance_absolute, int use_jacobi,
    const int32_t* tune_table, void* workspace, int64_t workspace_bytes,
    int32_t* iterations, double* residual_norms, void* stream, int32_t* tune_table_out);

/* ------------------------------------------ sparse products and sums -- */

/* C = A B (csr::spgemm, core/matrix/csr_kernels.hpp:72-76) and
 * C = alpha A B + beta D (csr::advanced_spgemm, :78-86), A num_rows x k,
 * B k x num_cols, int32 indices, in two calls because the caller owns C:
 * the symbolic call writes C's row pointers (num_rows + 1 entries) and its
 * entry count to *c_nnz (host); the caller allocates c_nnz columns and
 * values; the numeric call fills them.  D (and beta) are null for the plain
 * product; d_row_ptrs/d_col_idxs must then be null in the symbolic call too.
 * alpha and beta are device scalars (alpha may be null: 1).  Results are
 * bit-exact with the reference executor (reference/matrix/csr_kernels.cpp:
 * 199-300): columns ascending, each entry accumulated as beta d, then
 * + (alpha a_ik) b_kj over A's row in storage order, without fused
 * multiply-adds.  B's rows must not repeat a column.  Workspace:
 * b2s_csr_spgemm_workspace_bytes, the same for both calls. */
int64_t b2s_csr_spgemm_workspace_bytes(int64_t num_rows, int64_t num_cols);
int b2s_csr_spgemm_symbolic(int64_t num_rows, int64_t num_cols, const int32_t* a_row_ptrs,
                            const int32_t* a_col_idxs, const int32_t* b_row_ptrs,
                            const int32_t* b_col_idxs, const int32_t* d_row_ptrs,
                            const int32_t* d_col_idxs, int32_t* c_row_ptrs, int64_t* c_nnz,
                            void* workspace, int64_t workspace_bytes, void* stream);
int b2s_csr_spgemm_numeric_f64(int64_t num_rows, int64_t num_cols, const double* alpha,
                               const int32_t* a_row_ptrs, const int32_t* a_col_idxs,
                               const double* a_values, const int32_t* b_row_ptrs,
                               const int32_t* b_col_idxs, const double* b_values,
                               const double* beta, const int32_t* d_row_ptrs,
                               const int32_t* d_col_idxs, const double* d_values,
                               const int32_t* c_row_ptrs, int32_t* c_col_idxs,
                               double* c_values, void* workspace, int64_t workspace_bytes,
                               void* stream);
int b2s_csr_spgemm_numeric_f32(int64_t num_rows, int64_t num_cols, const float* alpha,
                               const int32_t* a_row_ptrs, const int32_t* a_col_idxs,
                               const float* a_values, const int32_t* b_row_ptrs,
                               const int32_t* b_col_idxs, const float* b_values,
                               const float* beta, const int32_t* d_row_ptrs,
                               const int32_t* d_col_idxs, const float* d_values,
                               const int32_t* c_row_ptrs, int32_t* c_col_idxs,
                               float* c_values, void* workspace, int64_t workspace_bytes,
                               void* stream);

/* C = alpha A + beta B for matrices with ascending columns in every row
 * (csr::spgeam, core/matrix/csr_kernels.hpp:88-93; reference/matrix/
 * csr_kernels.cpp:424-470): symbolic (C's row pointers, *c_nnz on the host)
 * then numeric; every column of either operand is stored, entries
 * alpha * a + beta * b with a missing side read as zero, bit-exact.
 * alpha, beta: device scalars. */
int64_t b2s_csr_spgeam_workspace_bytes(int64_t num_rows);
int b2s_csr_spgeam_symbolic(int64_t num_rows, const int32_t* a_row_ptrs,
                            const int32_t* a_col_idxs, const int32_t* b_row_ptrs,
                            const int32_t* b_col_idxs, int32_t* c_row_ptrs, int64_t* c_nnz,
                            void* workspace, int64_t workspace_bytes, void* stream);
int b2s_csr_spgeam_numeric_f64(int64_t num_rows, const double* alpha,
                               const int32_t* a_row_ptrs, const int32_t* a_col_idxs,
                               const double* a_values, const double* beta,
                               const int32_t* b_row_ptrs, const int32_t* b_col_idxs,
                               const double* b_values, const int32_t* c_row_ptrs,
                               int32_t* c_col_idxs, double* c_values, void* stream);
int b2s_csr_spgeam_numeric_f32(int64_t num_rows, const float* alpha,
                               const int32_t* a_row_ptrs, const int32_t* a_col_idxs,
                               const float* a_values, const float* beta,
                               const int32_t* b_row_ptrs, const int32_t* b_col_idxs,
                               const float* b_values, const int32_t* c_row_ptrs,
                               int32_t* c_col_idxs, float* c_values, void* stream);

/* ------------------------------------------------------------- Hybrid -- */

/* Csr -> Hybrid (csr::convert_to_hybrid, core/matrix/csr_kernels.hpp:
 * 106-110): the first ell_width entries of every row into the Ell part
 * (column-major, ell_stride >= num_rows, padding column -1 and value 0),
 * the rest into the Coo part in row order (coo_nnz entries, from
 * b2s_hybrid_config; a mismatch is B2S_ERR_INVALID_ARG).  Bit-exact. */
int64_t b2s_hybrid_convert_workspace_bytes(int64_t num_rows);
int b2s_csr_convert_to_hybrid_f64(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const double* values,
                                  int64_t ell_width, int64_t ell_stride,
                                  int32_t* ell_col_idxs, double* ell_values, int64_t coo_nnz,
                                  int32_t* coo_row_idxs, int32_t* coo_col_idxs,
                                  double* coo_values, void* workspace,
                                  int64_t workspace_bytes, void* stream);
int b2s_csr_convert_to_hybrid_f32(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const float* values,
                                  int64_t ell_width, int64_t ell_stride,
                                  int32_t* ell_col_idxs, float* ell_values, int64_t coo_nnz,
                                  int32_t* coo_row_idxs, int32_t* coo_col_idxs,
                                  float* coo_values, void* workspace,
                                  int64_t workspace_bytes, void* stream);

/* Hybrid SpMV (hybrid::spmv / advanced_spmv, core/matrix/hybrid_kernels.hpp:
 * the Ell part then the Coo part): per row, the Ell slots in order, then the
 * row's Coo entries in order (the Coo part sorted by row), c = A b or
 * alpha A b + beta c (beta == 0 ignores c). */
int b2s_hybrid_spmv_f64(int64_t num_rows, int64_t num_cols, int64_t ell_width,
                        int64_t ell_stride, const int32_t* ell_col_idxs,
                        const double* ell_values, int64_t coo_nnz,
                        const int32_t* coo_row_idxs, const int32_t* coo_col_idxs,
                        const double* coo_values, const double* b, int64_t ldb, double* c,
                        int64_t ldc, int64_t num_rhs, const double* alpha, const double* beta,
                        void* stream);
int b2s_hybrid_spmv_f32(int64_t num_rows, int64_t num_cols, int64_t ell_width,
                        int64_t ell_stride, const int32_t* ell_col_idxs,
                        const float* ell_values, int64_t coo_nnz,
                        const int32_t* coo_row_idxs, const int32_t* coo_col_idxs,
                        const float* coo_values, const float* b, int64_t ldb, float* c,
                        int64_t ldc, int64_t num_rhs, const float* alpha, const float* beta,
                        void* stream);

/* Hybrid -> Csr (Hybrid::convert_to(Csr), core/matrix/hybrid.cpp): row
 * pointers and the entry count (host) first, then the row's Ell entries
 * and Coo entries, columns sorted (stable). */
int b2s_hybrid_csr_row_ptrs(int64_t num_rows, int64_t ell_width, int64_t ell_stride,
                            const int32_t* ell_col_idxs, int64_t coo_nnz,
                            const int32_t* coo_row_idxs, int32_t* row_ptrs, int64_t* nnz,
                            void* workspace, int64_t workspace_bytes, void* stream);
int b2s_hybrid_convert_to_csr_f64(int64_t num_rows, int64_t ell_width, int64_t ell_stride,
                                  const int32_t* ell_col_idxs, const double* ell_values,
                                  int64_t coo_nnz, const int32_t* coo_row_idxs,
                                  const int32_t* coo_col_idxs, const double* coo_values,
                                  const int32_t* row_ptrs, int32_t* col_idxs, double* values,
                                  void* stream);
int b2s_hybrid_convert_to_csr_f32(int64_t num_rows, int64_t ell_width, int64_t ell_stride,
                                  const int32_t* ell_col_idxs, const float* ell_values,
                                  int64_t coo_nnz, const int32_t* coo_row_idxs,
                                  const int32_t* coo_col_idxs, const float* coo_values,
                                  const int32_t* row_ptrs, int32_t* col_idxs, float* values,
                                  void* stream);

/* ------------------------------------------------------- Hybrid set-up -- */
/* Ell width and Coo entry count of a Hybrid matrix (Ell + Coo) from its row
 * lengths, a HOST array, as the strategy classes compute them on the host
 * (include/ginkgo/core/matrix/hybrid.hpp:103-360, compute_hybrid_config):
 *   B2S_HYBRID_COLUMN_LIMIT          width = param1 (columns)
 *   B2S_HYBRID_IMBALANCE_LIMIT       the sorted row length at
 *                                    floor(rows * param1), param1 clamped to
 *                                    [0, 1] (the longest for 1)
 *   B2S_HYBRID_IMBALANCE_BOUNDED     min(imbalance_limit(param1),
 *                                    floor(rows * param2))
 *   B2S_HYBRID_MINIMAL_STORAGE       imbalance_limit(index_bytes /
 *                                    (value_bytes + 2 index_bytes))
 *   B2S_HYBRID_AUTOMATIC             imbalance_bounded(1/3, 0.001)
 * config_out: int64[2] = {width, coo entries}. */
#define B2S_HYBRID_COLUMN_LIMIT 0
#define B2S_HYBRID_IMBALANCE_LIMIT 1
#define B2S_HYBRID_IMBALANCE_BOUNDED 2
#define B2S_HYBRID_MINIMAL_STORAGE 3
#define B2S_HYBRID_AUTOMATIC 4
int b2s_hybrid_config(int64_t num_rows, const int64_t* row_nnz, int strategy,
                      double param1, double param2, int value_bytes,
                      int index_bytes, int64_t* config_out);

/* ------------------------------------------ MatrixMarket and binary I/O -- */
/* Host-side matrix data I/O: every pointer here is a HOST pointer and no
 * CUDA call is made.  Matrix data is the reference's matrix_data: a size
 * (rows x cols) and a list of (row, column, value) entries, 0-based.
 *
 * b2s_mtx_read parses num_bytes bytes as
 *   B2S_MTX_TEXT     MatrixMarket text: read_raw (core/base/mtx_io.cpp:
 *                    747-751, parser :53-742): layouts coordinate/array,
 *                    fields real/integer/pattern (complex is rejected for
 *                    real value types), modifiers general/symmetric/
 *                    skew-symmetric/hermitian expanded to both triangles;
 *   B2S_MTX_BINARY   the reference's binary format: read_binary_raw
 *                    (:882-927): a 32-byte header (magic "GINKGO" + value
 *                    and index type letters, rows, cols, entries as uint64)
 *                    then (row, col, value) records; file values double,
 *                    float, half or bfloat16, indices int32 or int64;
 *   B2S_MTX_GENERIC  text when the first byte is '%', else binary
 *                    (read_generic_raw, :930-941);
 * into value_type (B2S_MTX_F64 / B2S_MTX_F32) and index_type (B2S_MTX_I32 /
 * B2S_MTX_I64) entries sorted by (row, column) (matrix_data::
 * sort_row_major; entries with equal coordinates keep their file order).
 * *(void**)handle_out receives a handle that owns the result.
 *
 * b2s_mtx_write formats num_entries entries (in the given order) as
 *   B2S_MTX_COORDINATE  "%%MatrixMarket matrix coordinate real general",
 *   B2S_MTX_ARRAY       "%%MatrixMarket matrix array real general" (column-
 *                       major, absent entries written as 0),
 *   B2S_MTX_BINARY      the binary format (write_binary_raw, :943-978),
 * with text values printed as the reference's default stream format (six
 * significant digits); write_raw :980-1004.
 *
 * b2s_mtx_sizes writes int64[4] = {rows, cols, entries, bytes} of a handle
 * (bytes: the formatted output of a write, 0 after a read); b2s_mtx_copy
 * copies the entries (row_idxs/col_idxs of the handle's index type, values
 * of its value type) and/or the formatted bytes into caller arrays (any may
 * be NULL); b2s_mtx_free releases a handle.  Errors (malformed input, the
 * reference's StreamError cases) return B2S_ERR_INVALID_ARG with the
 * reference's message in b2s_last_error(). */
#define B2S_MTX_TEXT 0
#define B2S_MTX_BINARY 1
#define B2S_MTX_GENERIC 2
#define B2S_MTX_COORDINATE 3
#define B2S_MTX_ARRAY 4
#define B2S_MTX_F64 0
#define B2S_MTX_F32 1
#define B2S_MTX_I32 0
#define B2S_MTX_I64 1
int b2s_mtx_read(const void* bytes, int64_t num_bytes, int format, int value_type,
                 int index_type, void* handle_out);
int b2s_mtx_write(int64_t num_rows, int64_t num_cols, int64_t num_entries,
                  const void* row_idxs, const void* col_idxs, const void* values,
                  int value_type, int index_type, int format, void* handle_out);
int b2s_mtx_sizes(const void* handle, int64_t* sizes_out);
int b2s_mtx_copy(const void* handle, void* row_idxs, void* col_idxs, void* values,
                 void* bytes);
int b2s_mtx_free(void* handle);

#ifdef __cplusplus
}
#endif

#endif /* GINKGO_B200_H */
