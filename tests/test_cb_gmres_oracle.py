"""The CB-GMRES oracle (oracle/cb_gmres.py) against the reference's own CB-GMRES
solve tests (tests/golden/cb_gmres_cases.json), for every real value type and
storage precision the reference instantiates."""
import json
import os

import numpy as np
import pytest

from oracle import cb_gmres as CB

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "cb_gmres_cases.json")) as f:
    G = json.load(f)

_EPS = {"f64": np.finfo(np.float64).eps, "f32": np.finfo(np.float32).eps,
        "f16": np.finfo(np.float16).eps}
_RED1 = {"f64": "f32", "f32": "f16"}
_RED2 = {"f64": "f16", "f32": "f16"}


def _assert_precision(vt, storage):
    """assert_precision (reference/test/solver/cb_gmres_kernels.cpp:82-101)."""
    t = {"keep": vt, "integer": vt, "reduce1": _RED1[vt], "ireduce1": _RED1[vt],
         "reduce2": _RED2[vt], "ireduce2": _RED2[vt]}[storage]
    return 10 * _EPS[t]


def _rel_error(a, b):
    """get_relative_error (core/test/utils/assertions.hpp:275): Frobenius."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(a), np.linalg.norm(b))


PARAMS = [(c, vt, st) for c in G["cases"] for vt in ("f64", "f32") for st in G["storage"][vt]]


@pytest.mark.parametrize("case,vt,storage", PARAMS,
                         ids=[f"{c['name']}-{vt}-{st}" for c, vt, st in PARAMS])
def test_cb_gmres_oracle_meets_reference_known_answers(case, vt, storage):
    prec = None
    if "block_jacobi" in case:
        # Jacobi with max_block_size 3 (:508-510): blocks detected on the
        # Csr of A, the inverted blocks applied in the value type
        from oracle import jacobi as J
        A = np.array(case["A"])
        rp = np.arange(0, A.size + 1, A.shape[1])
        ci = np.tile(np.arange(A.shape[1]), A.shape[0])
        assert J.find_blocks(rp, ci, 3) == case["block_jacobi"]
        jac = J.generate(rp, ci, A.ravel(), 3, dtype=CB._FLOAT[vt])
        prec = lambda v: J.apply(jac, v)  # noqa: E731
    x, iters = CB.solve(case["A"], np.array(case["b"]), value_type=vt, storage=storage,
                        krylov_dim=case["krylov_dim"], max_iters=case["max_iters"],
                        preconditioner=prec)
    tol = _assert_precision(vt, storage)
    tol = np.sqrt(tol) if case.get("tol_sqrt") else case["tol_factor"] * tol
    err = _rel_error(x, case["x"])
    assert err <= tol, f"relative error {err:.3e} > {tol:.3e} after {iters} iterations"
