/*
 * CPU oracle for the sparse iterative-solve path — TEST INFRASTRUCTURE ONLY.
 * See oracle.h for what it restates and how it is pinned.  Built by
 * oracle/Makefile into oracle/_build/liboracle.so; only the tests, the smoke
 * check and the benchmark's CPU-baseline leg load it.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define T double
#define S f64
#include "oracle_t.inc"
#undef T
#undef S

#define T float
#define S f32
#include "oracle_t.inc"
#undef T
#undef S

/* reference/matrix/sellp_kernels.cpp:109-131: per-slice max row length
 * rounded up to stride_factor, then an exclusive prefix sum into slice_sets
 * (num_slices + 1 entries). */
void orc_sellp_compute_slice_sets(int64_t n, const int32_t* rp,
                                  int64_t slice_size, int64_t stride_factor,
                                  uint64_t* slice_sets,
                                  uint64_t* slice_lengths)
{
    int64_t num_slices = (n + slice_size - 1) / slice_size;
    for (int64_t s = 0; s < num_slices; ++s) {
        uint64_t len = 0;
        for (int64_t lr = 0; lr < slice_size; ++lr) {
            int64_t row = s * slice_size + lr;
            int64_t rl = row < n ? rp[row + 1] - rp[row] : 0;
            uint64_t padded =
                (uint64_t)((rl + stride_factor - 1) / stride_factor * stride_factor);
            if (padded > len) len = padded;
        }
        slice_lengths[s] = len;
    }
    uint64_t acc = 0;
    for (int64_t s = 0; s < num_slices; ++s) {
        slice_sets[s] = acc;
        acc += slice_lengths[s];
    }
    slice_sets[num_slices] = acc;
}

int64_t orc_csr_max_row_nnz(int64_t n, const int32_t* rp)
{
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t l = rp[i + 1] - rp[i];
        if (l > m) m = l;
    }
    return m;
}

/* Mixed-precision iterative refinement: FP64 residual r = b - A x and FP64
 * stop check ||r|| <= reduction ||b|| (core/solver/ir.cpp:225-256,
 * core/solver/update_residual.hpp:20-60); the correction solves A d = r with
 * GMRES on an FP32 copy of A (Csr::convert_to, core/matrix/csr.cpp:318-327),
 * FP32 vectors, zero initial guess, and x += d in FP64. */
int orc_ir_gmres_mixed(int64_t n, const int32_t* rp, const int32_t* ci,
                       const double* v, const double* b, double* x,
                       int krylov_dim, int inner_iters, double inner_reduction,
                       int max_outer, double reduction, int* outer_out,
                       int* inner_total_out, double* res_norm_out)
{
    int64_t nnz = rp[n];
    float* v32 = (float*)malloc(sizeof(float) * (size_t)nnz);
    float* inv32 = (float*)malloc(sizeof(float) * (size_t)n);
    float* r32 = (float*)malloc(sizeof(float) * (size_t)n);
    float* d32 = (float*)malloc(sizeof(float) * (size_t)n);
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t e = 0; e < nnz; ++e) v32[e] = (float)v[e];
    orc_jacobi_invert_diagonal_f32(n, rp, ci, v32, inv32);
    double one = 1, neg_one = -1, bnorm = 0, rnorm = 0;
    for (int64_t i = 0; i < n; ++i) bnorm += b[i] * b[i];
    bnorm = sqrt(bnorm);
    int outer, inner_total = 0, conv = 0;
    for (outer = 0;; ++outer) {
        memcpy(r, b, sizeof(double) * (size_t)n);
        orc_csr_spmv_f64(n, rp, ci, v, x, 1, r, 1, 1, &neg_one, &one);
        rnorm = 0;
        for (int64_t i = 0; i < n; ++i) rnorm += r[i] * r[i];
        rnorm = sqrt(rnorm);
        if (rnorm <= reduction * bnorm) { conv = 1; break; }
        if (outer >= max_outer) break;
        for (int64_t i = 0; i < n; ++i) {
            r32[i] = (float)r[i];
            d32[i] = 0.f;
        }
        int it = 0;
        double rn;
        orc_gmres_f32(n, rp, ci, v32, inv32, r32, d32, krylov_dim, 0, inner_iters,
                      inner_reduction, 0, &it, &rn);
        inner_total += it;
        for (int64_t i = 0; i < n; ++i) x[i] += (double)d32[i];
    }
    if (outer_out) *outer_out = outer;
    if (inner_total_out) *inner_total_out = inner_total;
    if (res_norm_out) *res_norm_out = rnorm;
    free(v32); free(inv32); free(r32); free(d32); free(r);
    return conv;
}
