"""Writes tests/golden/known_answers.json.

The cases are known-answer tests of the reference (Ginkgo 1.12), transcribed
by hand from its gtest sources; each carries the file:line it comes from.
Two cases ("cg_poisson_2d_256" below) hold results measured by running the
reference's Reference and OpenMP executors on the generated workload.
Run:  python tests/golden/make_known_answers.py
"""
import json
import math
import os

S2 = math.sqrt(2.0)
NAN = "nan"

# 2 x 3 matrix  [[1, 3, 2], [0, 5, 0]] shared by the Csr/Ell/Sellp tests
CSR_2X3 = {"n_rows": 2, "n_cols": 3, "row_ptrs": [0, 3, 4],
           "col_idxs": [0, 1, 2, 1], "values": [1.0, 3.0, 2.0, 5.0]}

cases = {
    "_about": __doc__.strip().splitlines()[0],
    "spmv": [
        {"name": "Csr.AppliesToDenseVector",
         "source": "reference/test/matrix/csr_kernels.cpp:353-362",
         "matrix": CSR_2X3, "x": [[2.0], [1.0], [4.0]],
         "expected": [[13.0], [5.0]]},
        {"name": "Csr.AppliesToDenseMatrix",
         "source": "reference/test/matrix/csr_kernels.cpp:414-426",
         "matrix": CSR_2X3, "x": [[2.0, 3.0], [1.0, -1.5], [4.0, 2.5]],
         "expected": [[13.0, 3.5], [5.0, -7.5]]},
        {"name": "Csr.AppliesLinearCombinationToDenseVector",
         "source": "reference/test/matrix/csr_kernels.cpp:505-518",
         "matrix": CSR_2X3, "x": [[2.0], [1.0], [4.0]], "y": [[1.0], [2.0]],
         "alpha": -1.0, "beta": 2.0, "expected": [[-11.0], [-1.0]]},
        {"name": "Csr.AppliesLinearCombinationToDenseVectorWithZeroBetaNaN",
         "source": "reference/test/matrix/csr_kernels.cpp:521-533",
         "matrix": CSR_2X3, "x": [[2.0], [1.0], [4.0]], "y": [[NAN], [NAN]],
         "alpha": -1.0, "beta": 0.0, "expected": [[-13.0], [-5.0]]},
        {"name": "Csr.AppliesLinearCombinationToDenseMatrix",
         "source": "reference/test/matrix/csr_kernels.cpp:590-607",
         "matrix": CSR_2X3, "x": [[2.0, 3.0], [1.0, -1.5], [4.0, 2.5]],
         "y": [[1.0, 0.5], [2.0, -1.5]], "alpha": -1.0, "beta": 2.0,
         "expected": [[-11.0, -2.5], [-1.0, 4.5]]},
    ],
    "convert_to_ell": {
        "name": "Csr.ConvertsToEll",
        "source": "reference/test/matrix/csr_kernels.cpp:1585-1595 with "
                  "assert_equal_to_mtx(const Ell*) :248-266",
        "matrix": CSR_2X3, "width": 3, "stride": 2,
        "col_idxs": [0, 1, 1, -1, 2, -1],
        "values": [1.0, 5.0, 3.0, 0.0, 2.0, 0.0]},
    "convert_to_sellp": {
        "name": "Csr.ConvertsToSellp",
        "source": "reference/test/matrix/csr_kernels.cpp:1251-1259 with "
                  "assert_equal_to_mtx(const Sellp*) :216-240",
        "matrix": CSR_2X3, "slice_size": 64, "stride_factor": 1,
        "slice_sets": [0, 3], "slice_lengths": [3],
        "checks": {"0": [0, 1.0], "1": [1, 5.0], "64": [1, 3.0],
                   "65": [-1, 0.0], "128": [2, 2.0], "129": [-1, 0.0]}},
    "sellp_slice2_stride2": {
        "name": "Sellp.AppliesWithSliceSizeAndStrideFactor*",
        "source": "reference/test/matrix/sellp_kernels.cpp:37-41,426-500",
        "matrix": CSR_2X3, "slice_size": 2, "stride_factor": 2,
        "x": [[2.0, 3.0], [1.0, -1.5], [4.0, 2.5]],
        "y": [[1.0, 0.5], [2.0, -1.5]], "alpha": -1.0, "beta": 2.0,
        "expected_simple": [[13.0, 3.5], [5.0, -7.5]],
        "expected_advanced": [[-11.0, -2.5], [-1.0, 4.5]]},
    "ell_stride16": {
        "name": "Ell mtx2 (stride 16)",
        "source": "reference/test/matrix/ell_kernels.cpp:37-43",
        "matrix": CSR_2X3, "stride": 16, "x": [[2.0], [1.0], [4.0]],
        "expected": [[13.0], [5.0]]},
    "transpose": [
        {"name": "Csr.SquareMtxIsTransposable",
         "source": "reference/test/matrix/csr_kernels.cpp:1612-1630",
         "dense": [[1.0, 3.0, 2.0], [0.0, 5.0, 0.0], [0.0, 1.5, 2.0]],
         "expected_dense": [[1.0, 0.0, 0.0], [3.0, 5.0, 1.5], [2.0, 0.0, 2.0]]},
        {"name": "Csr.NonSquareMtxIsTransposable",
         "source": "reference/test/matrix/csr_kernels.cpp:1634-1645",
         "dense": [[1.0, 3.0, 2.0], [0.0, 5.0, 0.0]],
         "expected_dense": [[1.0, 0.0], [3.0, 5.0], [2.0, 0.0]]},
    ],
    "cg_kernels": {
        "source": "reference/test/solver/cg_kernels.cpp:143-225",
        "step_1": {"p": 3.0, "z": -2.0, "rho": [2.0, 3.0],
                   "prev_rho": [8.0, 3.0], "stopped": [0, 1],
                   "expected_p": [[-1.25, 3.0], [-1.25, 3.0]]},
        "step_1_div_by_zero": {"p": 3.0, "z": -2.0, "rho": [1.0, 1.0],
                               "prev_rho": [0.0, 0.0], "stopped": [0, 0],
                               "expected_p": [[-2.0, -2.0], [-2.0, -2.0]]},
        "step_2": {"x": -2.0, "p": 3.0, "r": 4.0, "q": -5.0, "rho": [2.0, 3.0],
                   "beta": [8.0, 3.0], "stopped": [0, 1],
                   "expected_x": [[-1.25, -2.0], [-1.25, -2.0]],
                   "expected_r": [[5.25, 4.0], [5.25, 4.0]]},
        "step_2_div_by_zero": {"x": -2.0, "p": 3.0, "r": 4.0, "q": -5.0,
                               "rho": [1.0, 1.0], "beta": [0.0, 0.0],
                               "stopped": [0, 0],
                               "expected_x": [[-2.0, -2.0], [-2.0, -2.0]],
                               "expected_r": [[4.0, 4.0], [4.0, 4.0]]},
    },
    "solves": [
        {"name": "Cg.SolvesStencilSystem", "solver": "cg",
         "source": "reference/test/solver/cg_kernels.cpp:30-34,227-239",
         "dense": [[2, -1.0, 0.0], [-1.0, 2, -1.0], [0.0, -1.0, 2]],
         "b": [-1.0, 3.0, 1.0], "expected": [1.0, 3.0, 2.0],
         "max_iters": 400, "tol_factor": 1.0},
        {"name": "Cg.SolvesBigDenseSystem1", "solver": "cg",
         "source": "reference/test/solver/cg_kernels.cpp:45-52,419-435",
         "dense": [[8828.0, 2673.0, 4150.0, -3139.5, 3829.5, 5856.0],
                   [2673.0, 10765.5, 1805.0, 73.0, 1966.0, 3919.5],
                   [4150.0, 1805.0, 6472.5, 2656.0, 2409.5, 3836.5],
                   [-3139.5, 73.0, 2656.0, 6048.0, 665.0, -132.0],
                   [3829.5, 1966.0, 2409.5, 665.0, 4240.5, 4373.5],
                   [5856.0, 3919.5, 3836.5, -132.0, 4373.5, 5678.0]],
         "b": [1300083.0, 1018120.5, 906410.0, -42679.5, 846779.5, 1176858.5],
         "expected": [81.0, 55.0, 45.0, 5.0, 85.0, -10.0],
         "max_iters": 100, "tol_factor": 1e2},
        {"name": "Cg.SolvesBigDenseSystem2", "solver": "cg",
         "source": "reference/test/solver/cg_kernels.cpp:45-52,438-454",
         "dense": "Cg.SolvesBigDenseSystem1",
         "b": [886630.5, -172578.0, 684522.0, -65310.5, 455487.5, 607436.0],
         "expected": [33.0, -56.0, 81.0, -30.0, 21.0, 40.0],
         "max_iters": 100, "tol_factor": 1e2},
        {"name": "Bicgstab.SolvesDenseSystem", "solver": "bicgstab",
         "source": "reference/test/solver/bicgstab_kernels.cpp:31-34,410-421",
         "dense": [[1.0, -3.0, 0.0], [-4.0, 1.0, -3.0], [2.0, -1.0, 2.0]],
         "b": [-1.0, 3.0, 1.0], "expected": [-4.0, -1.0, 4.0],
         "max_iters": 8, "tol_factor": 1.0},
        {"name": "Gmres.SolvesStencilSystem", "solver": "gmres",
         "source": "reference/test/solver/gmres_kernels.cpp:41-53,433-444",
         "dense": [[1.0, 2.0, 3.0], [3.0, 2.0, -1.0], [0.0, -1.0, 2]],
         "b": [13.0, 7.0, 1.0], "expected": [1.0, 3.0, 2.0],
         "krylov_dim": 3, "max_iters": 4, "tol_factor": 1e1},
        {"name": "Gmres.SolvesBigDenseSystem1", "solver": "gmres",
         "source": "reference/test/solver/gmres_kernels.cpp:54-67,629-646",
         "dense": [[2295.7, -764.8, 1166.5, 428.9, 291.7, -774.5],
                   [2752.6, -1127.7, 1212.8, -299.1, 987.7, 786.8],
                   [138.3, 78.2, 485.5, -899.9, 392.9, 1408.9],
                   [-1907.1, 2106.6, 1026.0, 634.7, 194.6, -534.1],
                   [-365.0, -715.8, 870.7, 67.5, 279.8, 1927.8],
                   [-848.1, -280.5, -381.8, -187.1, 51.2, -176.2]],
         "b": [72748.36, 297469.88, 347229.24, 36290.66, 82958.82, -80192.15],
         "expected": [52.7, 85.4, 134.2, -250.0, -16.8, 35.3],
         "krylov_dim": 100, "max_iters": 100, "tol_factor": 1e3},
        {"name": "Gmres.SolvesBigDenseSystem2", "solver": "gmres",
         "source": "reference/test/solver/gmres_kernels.cpp:54-67,648-665",
         "dense": "Gmres.SolvesBigDenseSystem1",
         "b": [175352.10, 313410.50, 131114.10, -134116.30, 179529.30, -43564.90],
         "expected": [33.0, -56.0, 81.0, -30.0, 21.0, 40.0],
         "krylov_dim": 100, "max_iters": 100, "tol_factor": 1e3},
        # with a block Jacobi preconditioner of max_block_size 3, solved
        # with every ortho_method
        {"name": "Gmres.SolvesWithPreconditioner", "solver": "gmres",
         "source": "reference/test/solver/gmres_kernels.cpp:54-67,777-810",
         "dense": "Gmres.SolvesBigDenseSystem1",
         "b": [175352.10, 313410.50, 131114.10, -134116.30, 179529.30, -43564.90],
         "expected": [33.0, -56.0, 81.0, -30.0, 21.0, 40.0],
         "krylov_dim": 100, "max_iters": 100, "tol_factor": 1e3,
         "jacobi_block_size": 3},
        # tolerance sqrt(r) * 1e2 (half_tol), written as tol_sqrt
        {"name": "Gmres.SolvesBigDenseSystem1WithRestart", "solver": "gmres",
         "source": "reference/test/solver/gmres_kernels.cpp:77-82,750-775",
         "dense": [[-86.40, 153.30, -108.90, 8.60, -61.60],
                   [7.70, -77.00, 3.30, -149.20, 74.80],
                   [-121.40, 37.10, 55.30, -74.20, -19.20],
                   [-111.40, -22.60, 110.10, -106.20, 88.90],
                   [-0.70, 111.70, 154.40, 235.00, -76.50]],
         "b": [-13945.16, 11205.66, 16132.96, 24342.18, -10910.98],
         "expected": [-140.20, -142.20, 48.80, -17.70, -19.60],
         "krylov_dim": 4, "max_iters": 200, "tol_factor": 1e2, "tol_sqrt": True},
    ],
    # two right-hand sides solved together and one at a time: the combined
    # solve is at least as accurate as the single ones and matches them
    # within r (reference/test/solver/gmres_kernels.cpp:683-748)
    "gmres_multi_rhs": {
        "source": "reference/test/solver/gmres_kernels.cpp:54-67,683-748",
        "dense": "Gmres.SolvesBigDenseSystem1",
        "b1": [1300083.0, 1018120.5, 906410.0, -42679.5, 846779.5, 1176858.5],
        "b2": [886630.5, -172578.0, 684522.0, -65310.5, 455487.5, 607436.0],
        "krylov_dim": 100, "max_iters": 100},
    "gmres_kernels": {
        "source": "reference/test/solver/gmres_kernels.cpp:214-350",
        "hessenberg_qr_iter0": {
            "iteration": 0, "givens_cos": [[-0.5, 1.0], [70.0, -71.0]],
            "givens_sin": [[1.0, 0.0], [-72.0, 73.0]],
            "residual_norm_collection": [[1.25, 1.5], [NAN, NAN], [95.0, 94.0]],
            "hessenberg_iter": [[0.5, -0.75], [-0.5, 1.0], [97.0, 96.0]],
            "expected_givens_cos": [[0.5 * S2, -0.6], [70.0, -71.0]],
            "expected_givens_sin": [[-0.5 * S2, 0.8], [-72.0, 73.0]],
            "expected_hessenberg_iter": [[0.5 * S2, 1.25], [0.0, 0.0],
                                         [97.0, 96.0]],
            "expected_residual_norm_collection": [[0.625 * S2, -0.9],
                                                  [0.625 * S2, -1.2],
                                                  [95.0, 94.0]],
            "expected_residual_norm": [0.625 * S2, 1.2]},
        "hessenberg_qr_iter1": {
            "iteration": 1, "givens_cos": [[1.0, 0.5], [-0.5, 1.0]],
            "givens_sin": [[0.5, 0.25], [1.0, 0.0]],
            "residual_norm_collection": [[95.0, 94.0], [1.25, 1.5], [NAN, NAN]],
            "hessenberg_iter": [[-0.5, 4.0], [0.25, 0.5], [-0.5, 1.0]],
            "expected_givens_cos": [[1.0, 0.5], [0.5 * S2, -0.6]],
            "expected_givens_sin": [[0.5, 0.25], [-0.5 * S2, 0.8]],
            "expected_hessenberg_iter": [[-0.375, 2.125], [0.5 * S2, 1.25],
                                         [0.0, 0.0]],
            "expected_residual_norm_collection": [[95.0, 94.0],
                                                  [0.625 * S2, -0.9],
                                                  [0.625 * S2, -1.2]],
            "expected_residual_norm": [0.625 * S2, 1.2]},
        "solve_krylov": {
            "hessenberg": [[-1, 3, 0, 0, NAN, NAN], [2, -4, 1, 5, NAN, NAN]],
            "residual_norm_collection": [[12, 3], [-3, 15]],
            "expected_y": [[-18.0, 5.0], [-3.0, 3.0]]},
    },
    "batch_bicgstab": {
        "name": "BatchBicgstab.StencilSystemLoggerLogsIterations",
        "source": "reference/test/solver/batch_bicgstab_kernels.cpp:61-68,"
                  "124-141; core/test/utils/batch_helpers.hpp:95-121,211-234",
        "num_batch_items": 2, "num_rows": 15, "stencil": [-1.0, 6.0, -1.0],
        "exact_solution": 2.5, "tol": 5e-3, "max_iters": 100,
        "max_logged_iters": 5},
    "cg_poisson_2d_256": {
        "name": "CG + scalar Jacobi, 2D 5-point Poisson 256x256",
        "source": "measured with the reference's Reference and OpenMP "
                  "executors (libginkgo 1.12.0 built from source); x_true from "
                  "std::mt19937(1234) and std::uniform_real_distribution<double>"
                  "(-1, 1), b = A x_true, ResidualNorm(rhs_norm) 1e-10, "
                  "Iteration 1000",
        "grid": 256, "seed": 1234, "iterations": 710,
        "relative_residual": 9.777e-11},
}

out = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                   "known_answers.json")
with open(out, "w") as f:
    json.dump(cases, f, indent=1)
print("wrote", out)
