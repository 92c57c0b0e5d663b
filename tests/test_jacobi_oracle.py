"""The block Jacobi oracle (oracle/jacobi.py) against the reference's own
known answers (tests/golden/jacobi_cases.json, transcribed from
reference/test/preconditioner/jacobi_kernels.cpp), in FP64 and FP32."""
import json
import os

import numpy as np
import pytest

from oracle import jacobi as J

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "jacobi_cases.json")) as f:
    G = json.load(f)
MTX = G["dense"][0]["matrix"]
DT = [np.float64, np.float32]


def _csr(m):
    return np.array(m["row_ptrs"]), np.array(m["col_idxs"]), np.array(m["values"])


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = max(np.linalg.norm(a), np.linalg.norm(b))
    return 0.0 if den == 0 else np.linalg.norm(a - b) / den


@pytest.mark.parametrize("case", G["blocks"], ids=lambda c: c["name"])
def test_block_detection(case):
    rp, ci, _ = _csr(case["matrix"])
    got = case.get("block_ptrs") or J.find_blocks(rp, ci, case["max_block_size"])
    assert list(got) == case["expected"]


@pytest.mark.parametrize("dt", DT)
@pytest.mark.parametrize("case", G["dense"], ids=lambda c: c["name"])
def test_inverted_blocks(case, dt):
    rp, ci, v = _csr(case["matrix"])
    p = J.generate(rp, ci, v, case["max_block_size"], case.get("block_ptrs"),
                   case.get("aggregate_l1", False), dtype=dt)
    if case.get("transpose"):
        p = J.transpose(p)
    d = J.to_dense(p, len(rp) - 1)
    tol = 10 * np.finfo(dt).eps
    assert np.abs(d - np.array(case["expected"])).max() <= tol


@pytest.mark.parametrize("dt", DT)
@pytest.mark.parametrize("case", G["apply"], ids=lambda c: c["name"])
def test_apply(case, dt):
    rp, ci, v = _csr(MTX)
    p = J.generate(rp, ci, v, case["max_block_size"], case.get("block_ptrs"), dtype=dt)
    b = np.array(case["b"], dtype=dt)
    x = np.array(case["x"], dtype=dt)
    if "alpha" in case:
        got = J.apply(p, b, x, case["alpha"], case["beta"])
    else:
        got = J.apply(p, b)
    assert _rel(got, case["expected"]) <= 10 * np.finfo(dt).eps


@pytest.mark.parametrize("dt", DT)
@pytest.mark.parametrize("case", G["l1"], ids=lambda c: c["name"])
def test_l1_modifications(case, dt):
    rp, ci, v = _csr(case["matrix"])
    v = v.astype(dt)
    if case["kind"] == "scalar":
        diag = np.array([sum(v[k] for k in range(rp[r], rp[r + 1]) if ci[k] == r)
                         for r in range(len(rp) - 1)], dtype=dt)
        assert np.array_equal(J.scalar_l1(rp, ci, v, diag), np.array(case["expected"], dt))
    else:
        nv = J.block_l1(rp, ci, v, case["block_ptrs"])
        n = len(rp) - 1
        dense = np.zeros((n, n), dt)
        for r in range(n):
            for k in range(rp[r], rp[r + 1]):
                dense[r, ci[k]] = nv[k]
        assert np.array_equal(dense, np.array(case["expected"], dt))


def test_empty_matrix_has_no_blocks():
    # Jacobi.ConvertsEmptyToDense (reference/test/preconditioner/jacobi_kernels.cpp:1112-1121)
    p = J.generate(np.array([0]), np.array([], int), np.array([]), 32)
    assert J.to_dense(p, 0).shape == (0, 0)


@pytest.mark.parametrize("case", G["adaptive"], ids=lambda c: c["name"])
def test_adaptive_precision_known_answers(case):
    # the precisions each block ends with (value type double) and the
    # conditioning, as the reference's adaptive-precision tests state them
    m = case["matrix"]
    prec, chosen, conds = J.generate_adaptive(
        m["row_ptrs"], m["col_idxs"], m["values"], case["max_block_size"], case["block_ptrs"],
        accuracy=case.get("accuracy", 1e-1), precisions=case["precisions"])
    if "expected" in case:
        assert chosen == case["expected"]
    if "conditioning" in case:
        np.testing.assert_allclose(conds, case["conditioning"], rtol=1e-14)
    # every stored inverse is the full-precision inverse rounded to its
    # storage type and read back
    full = J.generate(m["row_ptrs"], m["col_idxs"], m["values"], case["max_block_size"],
                      block_ptrs=case["block_ptrs"])
    for blk, ref, p in zip(prec[2], full[2], chosen):
        np.testing.assert_array_equal(blk, J.storage_roundtrip(ref, p, np.float64))


def test_storage_types_round_values_as_the_reference():
    # truncated<double, 2> / <double, 4> keep the top 32 / 16 bits, truncated
    # <float, 2> the top 16 bits of the FP32 value, half goes through FP32
    # with values below its smallest normal flushed to zero
    x = np.array([1.0 / 3.0, -2.5e-5, 65519.0, 70000.0, -0.0])
    assert J.storage_roundtrip(x, J.P10, np.float64)[0] == np.float64(
        np.array([0x3FD5555500000000], np.uint64).view(np.float64)[0])
    assert J.storage_roundtrip(x, J.P20, np.float64)[0] == 0.328125
    assert J.storage_roundtrip(x, J.P11, np.float64)[0] == 0.33203125
    with np.errstate(over="ignore"):
        h = J.storage_roundtrip(x, J.P02, np.float64)
    assert h[0] == np.float64(np.float16(1.0 / 3.0))
    assert h[1] == 0.0 and np.signbit(h[1])
    assert h[2] == 65504.0 and np.isinf(h[3])
