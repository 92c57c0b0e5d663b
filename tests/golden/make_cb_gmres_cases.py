"""Writes tests/golden/cb_gmres_cases.json: the solve tests of the
reference's CB-GMRES (reference/test/solver/cb_gmres_kernels.cpp of Ginkgo
1.12), transcribed by hand with the file:line of each.

Every case runs for each real value type (double, float) and each storage
precision the reference instantiates for it (keep, reduce1, reduce2,
integer, ireduce1, ireduce2; TestTypes at :134-142).  The solver stops on
stop::Iteration(max_iters) or stop::ResidualNorm with the initial_resnorm
baseline and reduction factor r<T> = 10 eps(T) (:57-76); the expected
solution must be met to `tol_factor` x the storage's assert_precision (:82-101):
r<T> for keep and integer, r<reduce_precision<T>> for reduce1 and ireduce1,
r<reduce_precision<reduce_precision<T>>> for reduce2 and ireduce2
(`tol_sqrt`: the square root of that, as SolvesBigDenseSystem1WithRestart).
Run:  python tests/golden/make_cb_gmres_cases.py
"""
import json
import os

MTX = [[1.0, 2.0, 3.0], [3.0, 2.0, -1.0], [0.0, -1.0, 2.0]]          # :37-38
MTX2 = [[1.0, 2.0, 3.0], [4.0, 2.0, 1.0], [0.0, 1.0, 2.0]]          # :39-40
MTX_MEDIUM = [[-86.40, 153.30, -108.90, 8.60, -61.60],             # :41-47
              [7.70, -77.00, 3.30, -149.20, 74.80],
              [-121.40, 37.10, 55.30, -74.20, -19.20],
              [-111.40, -22.60, 110.10, -106.20, 88.90],
              [-0.70, 111.70, 154.40, 235.00, -76.50]]
MTX_BIG = [[2295.7, -764.8, 1166.5, 428.9, 291.7, -774.5],         # :48-55
           [2752.6, -1127.7, 1212.8, -299.1, 987.7, 786.8],
           [138.3, 78.2, 485.5, -899.9, 392.9, 1408.9],
           [-1907.1, 2106.6, 1026.0, 634.7, 194.6, -534.1],
           [-365.0, -715.8, 870.7, 67.5, 279.8, 1927.8],
           [-848.1, -280.5, -381.8, -187.1, 51.2, -176.2]]

cases = {
    "_about": __doc__.strip().splitlines()[0],
    "storage": {"f64": ["keep", "reduce1", "reduce2", "integer", "ireduce1", "ireduce2"],
                "f32": ["keep", "reduce1", "reduce2", "integer", "ireduce1", "ireduce2"]},
    "cases": [
        {"name": "CbGmres.SolvesStencilSystem",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:147-158",
         "A": MTX, "b": [[13.0], [7.0], [1.0]], "x": [[1.0], [3.0], [2.0]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 1},
        {"name": "CbGmres.SolvesStencilSystem2",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:224-246",
         "A": MTX2, "b": [[33.0], [20.0], [20.0]], "x": [[1.0], [4.0], [8.0]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 8},
        {"name": "CbGmres.SolvesMultipleStencilSystems",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:249-263",
         "A": MTX, "b": [[13.0, 6.0], [7.0, 4.0], [1.0, 1.0]],
         "x": [[1.0, 1.0], [3.0, 1.0], [2.0, 1.0]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 1},
        {"name": "CbGmres.SolvesBigDenseSystem1",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:372-386",
         "A": MTX_BIG,
         "b": [[72748.36], [297469.88], [347229.24], [36290.66], [82958.82], [-80192.15]],
         "x": [[52.7], [85.4], [134.2], [-250.0], [-16.8], [35.3]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 1},
        {"name": "CbGmres.SolvesBigDenseSystem2",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:389-403",
         "A": MTX_BIG,
         "b": [[175352.10], [313410.50], [131114.10], [-134116.30], [179529.30], [-43564.90]],
         "x": [[33.0], [-56.0], [81.0], [-30.0], [21.0], [40.0]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 1},
        {"name": "CbGmres.SolvesBigDenseSystem1WithRestart",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:474-498",
         "A": MTX_MEDIUM,
         "b": [[-13945.16], [11205.66], [16132.96], [24342.18], [-10910.98]],
         "x": [[-140.20], [-142.20], [48.80], [-17.70], [-19.60]],
         "max_iters": 200, "krylov_dim": 4, "tol_sqrt": True},
        {"name": "CbGmres.SolvesWithPreconditioner",
         "source": "reference/test/solver/cb_gmres_kernels.cpp:501-528",
         "A": MTX_BIG,
         "b": [[175352.10], [313410.50], [131114.10], [-134116.30], [179529.30], [-43564.90]],
         "x": [[33.0], [-56.0], [81.0], [-30.0], [21.0], [40.0]],
         "max_iters": 100, "krylov_dim": 100, "tol_factor": 4,
         "block_jacobi": [0, 3, 6]},
    ],
}

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "cb_gmres_cases.json"), "w") as f:
    json.dump(cases, f, indent=1)
    f.write("\n")
