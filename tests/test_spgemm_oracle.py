"""The SpGEMM / SpGEAM oracle (oracle/spgemm.py) against the reference's own
known answers (reference/test/matrix/csr_kernels.cpp; matrices transcribed
from its fixture at :84-190) and against dense products on random
matrices."""
import numpy as np
import pytest

from oracle import spgemm as S

# fixture (:84-106): 1 3 2 / 0 5 0
MTX = (np.array([0, 3, 4]), np.array([0, 1, 2, 1]), np.array([1.0, 3.0, 2.0, 5.0]))
# fixture (:108-131): 1 3 2 / {0} 5 0, an explicit zero kept
MTX2 = (np.array([0, 3, 5]), np.array([0, 1, 2, 0, 1]), np.array([1.0, 3.0, 2.0, 0.0, 5.0]))
# fixture (:133-190): 0 2 1 / 3 1 8 / 2 0 3, each row rotated once (unsorted)
MTX3_UNSORTED = (np.array([0, 2, 5, 7]), np.array([2, 1, 1, 2, 0, 2, 0]),
                 np.array([1.0, 2.0, 1.0, 8.0, 3.0, 3.0, 2.0]))


def _dense(m, n_cols):
    rp, ci, v = m
    d = np.zeros((len(rp) - 1, n_cols))
    for r in range(len(rp) - 1):
        for k in range(rp[r], rp[r + 1]):
            d[r, ci[k]] += v[k]
    return d


def _csr(d):
    rows = [np.nonzero(row)[0] for row in d]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
    ci = np.concatenate(rows) if rows else np.zeros(0, int)
    v = np.concatenate([d[i, r] for i, r in enumerate(rows)]) if rows else np.zeros(0)
    return rp, ci.astype(np.int64), v


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_multiplies_with_csr_matrix(dt):
    # Csr.AppliesToCsrMatrix / MultipliesWithCsrMatrix (:675-735): 13 5 31 / 15 5 40
    rp, ci, v = S.spgemm(MTX, MTX3_UNSORTED, dt)
    assert rp.tolist() == [0, 3, 6] and ci.tolist() == [0, 1, 2, 0, 1, 2]
    assert v.tolist() == [13, 5, 31, 15, 5, 40] and v.dtype == dt


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_applies_linear_combination_to_csr_matrix(dt):
    # Csr.AppliesLinearCombinationToCsrMatrix / MultiplyAddsWithCsrMatrices
    # (:772-841): -1 * mtx * mtx3 + 2 * mtx2 = -11 1 -27 / -15 5 -40
    rp, ci, v = S.advanced_spgemm(-1.0, MTX, MTX3_UNSORTED, 2.0, MTX2, dt)
    assert rp.tolist() == [0, 3, 6] and ci.tolist() == [0, 1, 2, 0, 1, 2]
    assert v.tolist() == [-11, 1, -27, -15, 5, -40]


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_scale_add_csr_matrices(dt):
    # Csr.ScaleAddCsrMatrices (:923-951): -3 a + 2 b on the union pattern
    a = np.array([[2, 0, 3], [0, 1, -1.5], [0, -2, 0], [5, 0, 0], [1, 0, 4], [2, -2, 0],
                  [0, 0, 0]])
    b = np.array([[2, -2, 0], [1, 0, 4], [2, 0, 3], [0, 1, -1.5], [1, 0, 0], [0, 0, 0],
                  [0, 0, 0]])
    exp = np.array([[-2, -4, -9], [2, -3, 12.5], [4, 6, 6], [-15, 2, -3], [-1, 0, -12],
                    [-6, 6, 0], [0, 0, 0]])
    rp, ci, v = S.spgeam(-3.0, _csr(a), 2.0, _csr(b), dt)
    erp, eci, _ = _csr(exp)
    assert rp.tolist() == erp.tolist() and ci.tolist() == eci.tolist()
    assert np.abs(_dense((rp, ci, v), 3) - exp).max() <= 10 * np.finfo(dt).eps * 15


def test_random_products_and_sums_match_dense():
    rng = np.random.default_rng(0)
    for _ in range(20):
        n, m, p = rng.integers(1, 30, size=3)
        A = np.where(rng.random((n, m)) < 0.2, rng.standard_normal((n, m)), 0.0)
        B = np.where(rng.random((m, p)) < 0.2, rng.standard_normal((m, p)), 0.0)
        D = np.where(rng.random((n, p)) < 0.2, rng.standard_normal((n, p)), 0.0)
        C = S.spgemm(_csr(A), _csr(B))
        assert np.allclose(_dense(C, p), A @ B, atol=1e-12)
        assert all(np.all(np.diff(C[1][C[0][r]:C[0][r + 1]]) > 0) for r in range(n))
        C = S.advanced_spgemm(0.5, _csr(A), _csr(B), -2.0, _csr(D))
        assert np.allclose(_dense(C, p), 0.5 * A @ B - 2.0 * D, atol=1e-12)
        E = np.where(rng.random((n, p)) < 0.3, rng.standard_normal((n, p)), 0.0)
        C = S.spgeam(1.5, _csr(D), -0.5, _csr(E))
        assert np.allclose(_dense(C, p), 1.5 * D - 0.5 * E, atol=1e-12)
        # union pattern: a column stored in either input is stored in the sum
        for r in range(n):
            want = sorted(set(np.nonzero(D[r])[0]) | set(np.nonzero(E[r])[0]))
            assert C[1][C[0][r]:C[0][r + 1]].tolist() == want


def test_hybrid_conversions_match_reference_known_answers():
    # Csr.ConvertsToHybridAutomatically (reference/test/matrix/csr_kernels.cpp:
    # 1301-1309, assert_equal_to_mtx :277-298): automatic -> Ell width 0
    rp, ci, v = MTX
    w = S.hybrid_width(np.diff(rp), "automatic")
    h = S.csr_to_hybrid(rp, ci, v, w)
    assert w == 0 and h["stride"] == 2
    assert h["coo_row_idxs"].tolist() == [0, 0, 0, 1]
    assert h["coo_col_idxs"].tolist() == [0, 1, 2, 1]
    assert h["coo_values"].tolist() == [1.0, 3.0, 2.0, 5.0]
    # Csr.ConvertsToHybridByColumn2 (:1326-1336, assert_equal_to_mtx2 :300-330)
    rp, ci, v = MTX2
    h = S.csr_to_hybrid(rp, ci, v, S.hybrid_width(np.diff(rp), "column_limit", num_columns=2))
    assert h["width"] == 2 and h["stride"] == 2
    assert h["ell_values"].tolist() == [1, 0, 3, 5] and h["ell_col_idxs"].tolist() == [0, 0, 1, 1]
    assert h["coo_row_idxs"].tolist() == [0] and h["coo_col_idxs"].tolist() == [2]
    assert h["coo_values"].tolist() == [2.0]


def test_hybrid_apply_and_back_to_csr_known_answers():
    # Hybrid.AppliesToDenseVector / AppliesToDenseMatrix (reference/test/matrix/
    # hybrid_kernels.cpp:102-145) on mtx3 (:40-65): Ell width 2, one Coo entry
    h = {"rows": 2, "width": 2, "stride": 2,
         "ell_values": np.array([1.0, 0.0, 3.0, 5.0]),
         "ell_col_idxs": np.array([0, -1, 1, 1]),
         "coo_row_idxs": np.array([0]), "coo_col_idxs": np.array([2]),
         "coo_values": np.array([2.0])}
    assert S.hybrid_apply(h, np.array([2.0, 1.0, 4.0])).tolist() == [13.0, 5.0]
    y = S.hybrid_apply(h, np.array([[2.0, 3.0], [1.0, -1.5], [4.0, 2.5]]))
    assert y.tolist() == [[13.0, 3.5], [5.0, -7.5]]
    # ConvertsToCsr (:307-322): 1 3 2 / 0 5 0 with sorted columns
    rp, ci, v = S.hybrid_to_csr(h)
    assert rp.tolist() == [0, 3, 4] and ci.tolist() == [0, 1, 2, 1]
    assert v.tolist() == [1.0, 3.0, 2.0, 5.0]


def test_hybrid_strategies_and_round_trip_on_random_rows():
    rng = np.random.default_rng(3)
    for _ in range(10):
        n, m = int(rng.integers(1, 200)), 300
        lens = rng.integers(0, 12, size=n)
        rows = [np.sort(rng.choice(m, size=k, replace=False)) for k in lens]
        rp = np.concatenate([[0], np.cumsum(lens)])
        ci = np.concatenate(rows).astype(np.int64) if rows else np.zeros(0, np.int64)
        v = rng.standard_normal(len(ci))
        x = rng.standard_normal(m)
        dense = _dense((rp, ci, v), m)
        for strat, kw in (("automatic", {}), ("imbalance_limit", {"percent": 0.5}),
                          ("imbalance_bounded_limit", {"percent": 0.9, "ratio": 0.05}),
                          ("minimal_storage_limit", {}), ("column_limit", {"num_columns": 3})):
            w = S.hybrid_width(lens, strat, **kw)
            h = S.csr_to_hybrid(rp, ci, v, w)
            assert len(h["coo_values"]) == sum(max(0, k - w) for k in lens)
            np.testing.assert_allclose(S.hybrid_apply(h, x), dense @ x, atol=1e-12)
            back = S.hybrid_to_csr(h)
            assert back[0].tolist() == rp.tolist() and back[1].tolist() == ci.tolist()
            assert np.array_equal(back[2], v)


@pytest.mark.parametrize("strategy,kw,width,ell_c,ell_v,coo", [
    # core/test/matrix/hybrid.cpp:170-200 (automatic), :203-211 with
    # assert_equal_to_original_mtx :62-86 (column_limit 2), :214-244 (imbalance 0.4)
    ("automatic", {}, 0, [], [], ([0, 0, 0, 1], [0, 1, 2, 1], [1.0, 0.0, 2.0, 5.0])),
    ("column_limit", {"num_columns": 2}, 2, [0, 1, 1, -1], [1.0, 5.0, 0.0, 0.0],
     ([0], [2], [2.0])),
    ("imbalance_limit", {"percent": 0.4}, 1, [0, 1], [1.0, 5.0],
     ([0, 0], [1, 2], [0.0, 2.0])),
])
def test_hybrid_read_known_answers(strategy, kw, width, ell_c, ell_v, coo):
    # matrix data {(0,0,1), (0,1,0), (0,2,2), (1,1,5)}: the explicit zero is stored
    rp, ci, v = np.array([0, 3, 4]), np.array([0, 1, 2, 1]), np.array([1.0, 0.0, 2.0, 5.0])
    w = S.hybrid_width(np.diff(rp), strategy, **kw)
    h = S.csr_to_hybrid(rp, ci, v, w)
    assert w == width and h["stride"] == 2
    assert h["ell_col_idxs"].tolist() == ell_c and h["ell_values"].tolist() == ell_v
    assert (h["coo_row_idxs"].tolist(), h["coo_col_idxs"].tolist(),
            h["coo_values"].tolist()) == coo
