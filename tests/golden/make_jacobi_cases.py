"""Writes tests/golden/jacobi_cases.json: known answers of the reference's
block Jacobi tests (reference/test/preconditioner/jacobi_kernels.cpp of
Ginkgo 1.12), transcribed by hand with the file:line of each.  Real value
types, full-precision blocks (the adaptive-precision cases are not kept).
Tolerance r<T> = 10 eps(T) unless a case says otherwise.
Run:  python tests/golden/make_jacobi_cases.py
"""
import json
import os

# fixture matrix (:64-78):   4 -2 . . -2 / -1 4 . . . / . . 4 -2 . /
#                            . . -1 4 -2 / -1 . . -1 4
MTX = {"row_ptrs": [0, 3, 5, 7, 10, 13],
       "col_idxs": [0, 1, 4, 0, 1, 2, 3, 2, 3, 4, 0, 3, 4],
       "values": [4.0, -2.0, -2.0, -1.0, 4.0, 4.0, -2.0, -1.0, 4.0, -2.0, -1.0, -1.0, 4.0]}
INV_DENSE = [[4 / 14, 2 / 14, 0, 0, 0], [1 / 14, 4 / 14, 0, 0, 0],
             [0, 0, 14 / 48, 8 / 48, 4 / 48], [0, 0, 4 / 48, 16 / 48, 8 / 48],
             [0, 0, 1 / 48, 4 / 48, 14 / 48]]
X1 = [[1.0], [-1.0], [2.0], [-2.0], [3.0]]
B1 = [[4.0], [-1.0], [-2.0], [4.0], [-1.0]]
X2 = [[1.0, 0.5], [-1.0, -0.5], [2.0, 1.0], [-2.0, -1.0], [3.0, 1.5]]
B2 = [[4.0, -2.0], [-1.0, 4.0], [-2.0, 0.0], [4.0, -2.0], [-1.0, 4.0]]
SRC = "reference/test/preconditioner/jacobi_kernels.cpp"
# r<double> (core/test/utils.hpp:388-400): 10 epsilon of double, and its root
R = 10 * 2.0 ** -52
HALF_TOL = R ** 0.5

cases = {
    "_about": __doc__.strip().splitlines()[0],
    "blocks": [
        {"name": "Jacobi.CanBeGenerated", "source": SRC + ":94-107", "matrix": MTX,
         "max_block_size": 3, "block_ptrs": [0, 2, 5], "expected": [0, 2, 5]},
        {"name": "Jacobi.FindsNaturalBlocks", "source": SRC + ":129-156",
         "matrix": {"row_ptrs": [0, 2, 4, 6, 8], "col_idxs": [0, 1, 0, 1, 0, 2, 0, 2],
                    "values": [1.0] * 8}, "max_block_size": 3, "expected": [0, 2, 4]},
        {"name": "Jacobi.ExecutesSupervariableAgglomeration", "source": SRC + ":159-188",
         "matrix": {"row_ptrs": [0, 2, 4, 6, 8, 9], "col_idxs": [0, 1, 0, 1, 2, 3, 2, 3, 4],
                    "values": [1.0] * 9}, "max_block_size": 3, "expected": [0, 2, 5]},
        {"name": "Jacobi.AdheresToBlockSizeBound", "source": SRC + ":191-223",
         "matrix": {"row_ptrs": [0, 1, 2, 3, 4, 5, 6, 7], "col_idxs": [0, 1, 2, 3, 4, 5, 6],
                    "values": [1.0] * 7}, "max_block_size": 3, "expected": [0, 3, 6, 7]},
        {"name": "Jacobi.CanBeGeneratedWithUnknownBlockSizes", "source": SRC + ":226-241",
         "matrix": MTX, "max_block_size": 3, "expected": [0, 3, 5]},
    ],
    "dense": [
        {"name": "Jacobi.InvertsDiagonalBlocks", "source": SRC + ":244-267",
         "matrix": MTX, "max_block_size": 3, "block_ptrs": [0, 2, 5], "expected": INV_DENSE},
        {"name": "Jacobi.CanTransposeDiagonalBlocks", "source": SRC + ":301-326",
         "matrix": MTX, "max_block_size": 3, "block_ptrs": [0, 2, 5], "transpose": True,
         "expected": [list(r) for r in zip(*INV_DENSE)]},
        {"name": "Jacobi.PivotsWhenInvertingBlocks", "source": SRC + ":452-490",
         "matrix": {"row_ptrs": [0, 3, 6, 9], "col_idxs": [0, 1, 2, 0, 1, 2, 0, 1, 2],
                    "values": [0.0, 2.0, 0.0, 0.0, 0.0, 4.0, 1.0, 0.0, 0.0]},
         "max_block_size": 3, "block_ptrs": [0, 3],
         "expected": [[0.0, 0.0, 1.0], [0.5, 0.0, 0.0], [0.0, 0.25, 0.0]]},
        {"name": "Jacobi.ConvertsToDense", "source": SRC + ":1073-1089",
         "matrix": MTX, "max_block_size": 3, "block_ptrs": [0, 2, 5], "expected": INV_DENSE},
        {"name": "Jacobi.L1BlockJaocbiConvertsToDense", "source": SRC + ":1187-1228",
         "matrix": {"row_ptrs": [0, 3, 5, 7, 10, 12],
                    "col_idxs": [0, 1, 4, 0, 1, 2, 3, 2, 3, 4, 0, 3],
                    "values": [2.0, -2.0, -2.0, -1.0, 4.0, 4.0, -2.0, -1.0, 4.0, -2.0, -4.0, -1.0]},
         "max_block_size": 3, "block_ptrs": [0, 2, 5], "aggregate_l1": True,
         "expected": INV_DENSE},
    ],
    "apply": [
        {"name": "Jacobi.AppliesToVector", "source": SRC + ":627-638", "max_block_size": 3,
         "block_ptrs": [0, 2, 5], "x": X1, "b": B1,
         "expected": [[1.0], [0.0], [0.0], [1.0], [0.0]]},
        {"name": "Jacobi.ScalarJacobiAppliesToVector", "source": SRC + ":641-653",
         "max_block_size": 1, "x": X1, "b": B1,
         "expected": [[1.0], [-0.25], [-0.5], [1.0], [-0.25]]},
        {"name": "Jacobi.AppliesToMultipleVectors", "source": SRC + ":758-780",
         "max_block_size": 3, "block_ptrs": [0, 2, 5], "x": X2, "b": B2,
         "expected": [[1.0, 0.0], [0.0, 1.0], [0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]},
        {"name": "Jacobi.ScalarJacobiAppliesToMultipleVectors", "source": SRC + ":783-806",
         "max_block_size": 1, "x": X2, "b": B2,
         "expected": [[1.0, -0.5], [-0.25, 1.0], [-0.5, 0.0], [1.0, -0.5], [-0.25, 1.0]]},
        {"name": "Jacobi.AppliesLinearCombinationToVector", "source": SRC + ":868-882",
         "max_block_size": 3, "block_ptrs": [0, 2, 5], "x": X1, "b": B1, "alpha": 2.0,
         "beta": -1.0, "expected": [[1.0], [1.0], [-2.0], [4.0], [-3.0]]},
        {"name": "Jacobi.ScalarJacobiAppliesLinearCombinationToVector",
         "source": SRC + ":885-899", "max_block_size": 1, "x": X1, "b": B1, "alpha": 2.0,
         "beta": -1.0, "expected": [[1.0], [0.5], [-3.0], [4.0], [-3.5]]},
        {"name": "Jacobi.AppliesLinearCombinationToMultipleVectors",
         "source": SRC + ":988-1013", "max_block_size": 3, "block_ptrs": [0, 2, 5],
         "x": X2, "b": B2, "alpha": 2.0, "beta": -1.0,
         "expected": [[1.0, -0.5], [1.0, 2.5], [-2.0, -1.0], [4.0, 1.0], [-3.0, 0.5]]},
        {"name": "Jacobi.ScalarAppliesLinearCombinationToMultipleVectors",
         "source": SRC + ":1016-1041", "max_block_size": 1, "x": X2, "b": B2,
         "alpha": 2.0, "beta": -1.0,
         "expected": [[1.0, -1.5], [0.5, 2.5], [-3.0, -1.0], [4.0, 0.0], [-3.5, 0.5]]},
    ],
    "l1": [
        {"name": "Jacobi.ScalarL1Diag", "source": SRC + ":1124-1151", "kind": "scalar",
         "matrix": {"row_ptrs": [0, 2, 4, 6, 8], "col_idxs": [0, 1, 0, 1, 0, 2, 0, 2],
                    "values": [1.0, 1.0, 2.0, 2.0, -5.0, 1.0, 1.0, -1.0]},
         "expected": [2.0, 4.0, 6.0, 2.0]},
        {"name": "Jacobi.BlockL1", "source": SRC + ":1154-1184", "kind": "block",
         "matrix": {"row_ptrs": [0, 2, 4, 6, 9], "col_idxs": [0, 1, 0, 1, 0, 2, 0, 2, 3],
                    "values": [1.0, 1.0, 2.0, 2.0, -5.0, 1.0, 1.0, -1.0, 1.0]},
         "block_ptrs": [0, 1, 2, 4],
         "expected": [[2.0, 1.0, 0.0, 0.0], [2.0, 4.0, 0.0, 0.0], [-5.0, 0.0, 6.0, 0.0],
                      [1.0, 0.0, -1.0, 2.0]]},
    ],
    # adaptive precision (storage_optimization): the precisions each block
    # ends with (precision_reduction's byte, (preserving << 4) | nonpreserving,
    # 255 = autodetect) for value type double, the conditioning, and the
    # stored inverses as the tests read them back.  R = r<double> = 10 eps
    "adaptive": [
        {"name": "Jacobi.CanBeGeneratedWithAdaptivePrecision",
         "source": SRC + ":35-62,110-127", "matrix": MTX, "max_block_size": 17,
         "block_ptrs": [0, 2, 5], "precisions": [0x01, 0x00], "expected": [0x01, 0x00]},
        {"name": "Jacobi.ComputesConditioning", "source": SRC + ":535-548",
         "matrix": MTX, "max_block_size": 17, "block_ptrs": [0, 2, 5],
         "precisions": [0x01, 0x00], "conditioning": [6.0 * 6.0 / 14.0, 7.0 * 28.0 / 48.0]},
        {"name": "Jacobi.InvertsDiagonalBlocksWithAdaptivePrecisionAndSmallBlocks",
         "source": SRC + ":419-448", "matrix": MTX, "max_block_size": 3,
         "block_ptrs": [0, 2, 5], "precisions": [0x01, 0x00], "expected": [0x00, 0x00]},
        {"name": "Jacobi.SelectsCorrectBlockPrecisions", "source": SRC + ":551-578",
         "matrix": MTX, "max_block_size": 17, "block_ptrs": [0, 2, 5], "precisions": None,
         "accuracy": 1.5e-3, "expected": [0x02, 0x01]},
        {"name": "Jacobi.AvoidsPrecisionsThatOverflow", "source": SRC + ":581-623",
         "matrix": {"row_ptrs": [0, 2, 4, 6, 8], "col_idxs": [0, 1, 0, 1, 2, 3, 2, 3],
                    "values": [2.0, 1.0, 1.0, 2.0, HALF_TOL, -R, R, HALF_TOL]},
         "max_block_size": 13, "block_ptrs": [0, 2, 4], "precisions": None,
         "accuracy": 1e-1, "expected": [0x11, 0x11]},
    ],
}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "jacobi_cases.json"), "w") as f:
    json.dump(cases, f, indent=1)
    f.write("\n")
