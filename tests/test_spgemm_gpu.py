"""SpGEMM, SpGEAM and the Hybrid format on the GPU against the oracle
(oracle/spgemm.py, a restatement of the reference executor) and the
reference's known answers (reference/test/matrix/csr_kernels.cpp,
hybrid_kernels.cpp).  Patterns, columns and values are bit-exact: the device
accumulates every entry in the reference's order with its roundings."""
import numpy as np
import pytest
import torch

from ginkgo_b200.matrix import Csr, CudaExecutor, Identity, spgeam, spgemm
from oracle import spgemm as S

pytestmark = pytest.mark.gpu

NP = {torch.float64: np.float64, torch.float32: np.float32}
DTS = [torch.float64, torch.float32]

# the reference fixtures (csr_kernels.cpp:84-190)
MTX = (np.array([0, 3, 4]), np.array([0, 1, 2, 1]), np.array([1.0, 3.0, 2.0, 5.0]))
MTX2 = (np.array([0, 3, 5]), np.array([0, 1, 2, 0, 1]), np.array([1.0, 3.0, 2.0, 0.0, 5.0]))
MTX3_UNSORTED = (np.array([0, 2, 5, 7]), np.array([2, 1, 1, 2, 0, 2, 0]),
                 np.array([1.0, 2.0, 1.0, 8.0, 3.0, 3.0, 2.0]))


@pytest.fixture(scope="module")
def exe():
    return CudaExecutor.create(0)


def dev(exe, m, shape, dt):
    rp, ci, v = m
    return Csr(exe, shape, torch.tensor(np.asarray(rp), dtype=torch.int32),
               torch.tensor(np.asarray(ci), dtype=torch.int32),
               torch.tensor(np.asarray(v, dtype=NP[dt])))


def host(C):
    return (C.row_ptrs.cpu().numpy(), C.col_idxs.cpu().numpy(), C.values.cpu().numpy())


def assert_same(C, ref, what=""):
    rp, ci, v = host(C)
    assert rp.tolist() == np.asarray(ref[0]).tolist(), what
    assert ci.tolist() == np.asarray(ref[1]).tolist(), what
    assert v.dtype == np.asarray(ref[2]).dtype
    np.testing.assert_array_equal(v, ref[2], err_msg=what)


@pytest.mark.parametrize("dt", DTS)
def test_known_answers(exe, dt):
    A = dev(exe, MTX, (2, 3), dt)
    B = dev(exe, MTX3_UNSORTED, (3, 3), dt)
    # Csr.AppliesToCsrMatrix (:675-735): 13 5 31 / 15 5 40, through apply
    Cm = dev(exe, MTX2, (2, 3), dt)
    A.apply(B, Cm)
    assert_same(Cm, ([0, 3, 6], [0, 1, 2, 0, 1, 2],
                     np.array([13, 5, 31, 15, 5, 40], NP[dt])))
    # Csr.AppliesLinearCombinationToCsrMatrix (:772-841): -mtx mtx3 + 2 mtx2
    D = dev(exe, MTX2, (2, 3), dt)
    A.apply(-1.0, B, 2.0, D)
    assert_same(D, ([0, 3, 6], [0, 1, 2, 0, 1, 2],
                    np.array([-11, 1, -27, -15, 5, -40], NP[dt])))
    # Csr.ScaleAddCsrMatrices (:923-951): -3 a + 2 b on the union pattern
    a = np.array([[2, 0, 3], [0, 1, -1.5], [0, -2, 0], [5, 0, 0], [1, 0, 4], [2, -2, 0],
                  [0, 0, 0]])
    b = np.array([[2, -2, 0], [1, 0, 4], [2, 0, 3], [0, 1, -1.5], [1, 0, 0], [0, 0, 0],
                  [0, 0, 0]])

    def csr(d):
        rows = [np.nonzero(r)[0] for r in d]
        rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
        return rp, np.concatenate(rows), np.concatenate([d[i, r] for i, r in enumerate(rows)])
    Ad, Bd = dev(exe, csr(a), (7, 3), dt), dev(exe, csr(b), (7, 3), dt)
    Ad.apply(-3.0, Identity(3), 2.0, Bd)
    ref = S.spgeam(-3.0, csr(a), 2.0, csr(b), NP[dt])
    assert_same(Bd, ref)


def random_csr(rng, n, m, lens, sort=True, dtype=np.float64):
    """Rows of the given lengths, distinct random columns (sorted unless
    sort is False), values ~ N(0, 1) rounded to dtype."""
    rows = [rng.choice(m, size=int(k), replace=False) for k in lens]
    if sort:
        rows = [np.sort(r) for r in rows]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    ci = np.concatenate(rows).astype(np.int64) if len(rows) else np.zeros(0, np.int64)
    return rp, ci, rng.standard_normal(len(ci)).astype(dtype)


@pytest.mark.parametrize("dt", DTS)
@pytest.mark.parametrize("sort_b", [True, False])
def test_random_products_every_bin(exe, dt, sort_b):
    """Rows of every size class: short products (warp), a few hundred
    candidates (block) and rows of more than 8192 candidates (bitmap);
    empty rows; B's rows unsorted in one variant."""
    rng = np.random.default_rng(5 + int(sort_b))
    n, k, m = 1500, 1200, 20000
    lens_a = rng.integers(0, 12, size=n)
    lens_a[rng.choice(n, 30, replace=False)] = 60     # 60 x ~35: block bin
    lens_a[rng.choice(n, 6, replace=False)] = 400     # 400 x ~35: bitmap bin
    lens_a[:5] = 0
    lens_b = rng.integers(0, 70, size=k)
    a = random_csr(rng, n, k, lens_a, dtype=NP[dt])
    b = random_csr(rng, k, m, lens_b, sort=sort_b, dtype=NP[dt])
    ub = np.array([lens_b[a[1][a[0][r]:a[0][r + 1]]].sum() for r in range(n)])
    assert (ub > 8192).any() and ((ub > 512) & (ub <= 8192)).any() and (ub <= 512).any()
    A, B = dev(exe, a, (n, k), dt), dev(exe, b, (k, m), dt)
    ref = S.spgemm(a, b, NP[dt])
    assert_same(spgemm(A, B), ref, "spgemm")
    # advanced, D with its own pattern
    d = random_csr(rng, n, m, rng.integers(0, 20, size=n), dtype=NP[dt])
    D = dev(exe, d, (n, m), dt)
    ref = S.advanced_spgemm(0.75, a, b, -1.5, d, NP[dt])
    assert_same(spgemm(A, B, alpha=0.75, beta=-1.5, d=D), ref, "advanced_spgemm")


@pytest.mark.parametrize("dt", DTS)
def test_random_sums(exe, dt):
    rng = np.random.default_rng(8)
    n, m = 5000, 3000
    a = random_csr(rng, n, m, rng.integers(0, 40, size=n), dtype=NP[dt])
    b = random_csr(rng, n, m, rng.integers(0, 40, size=n), dtype=NP[dt])
    A, B = dev(exe, a, (n, m), dt), dev(exe, b, (n, m), dt)
    assert_same(spgeam(1.25, A, -0.5, B), S.spgeam(1.25, a, -0.5, b, NP[dt]))
    # cancellation keeps the entry (a - a)
    z = spgeam(1.0, A, -1.0, A)
    assert z.nnz == A.nnz and torch.count_nonzero(z.values) == 0


def test_product_of_poisson_stencil(exe):
    """A^2 of the 2D 5-point Poisson matrix: 13-point rows."""
    from ginkgo_b200 import stencils
    rp, ci, v = stencils.poisson_2d_5pt(200)
    A = dev(exe, (rp, ci, v), (len(rp) - 1,) * 2, torch.float64)
    C = spgemm(A, A)
    ref = S.spgemm((rp, ci, v), (rp, ci, v))
    assert_same(C, ref)


@pytest.mark.parametrize("dt", DTS)
def test_hybrid_known_answers(exe, dt):
    # Hybrid.AppliesToDenseVector / Matrix (hybrid_kernels.cpp:102-145) on
    # mtx3 with column limit 2 (Ell 1 3 / 0 5, Coo (0, 2, 2))
    A = dev(exe, MTX, (2, 3), dt)
    H = A.convert_to_hybrid("column_limit", num_columns=2)
    assert H.width == 2 and H.coo_nnz == 1
    assert H.ell_col_idxs.cpu().tolist() == [0, 1, 1, -1]
    assert H.coo_col_idxs.cpu().tolist() == [2]
    x = torch.tensor([[2.0, 3.0], [1.0, -1.5], [4.0, 2.5]], dtype=dt, device="cuda")
    y = torch.empty((2, 2), dtype=dt, device="cuda")
    H.apply(x, y)
    assert y.cpu().tolist() == [[13.0, 3.5], [5.0, -7.5]]
    # back to Csr (hybrid_kernels.cpp:307-322)
    assert_same(H.convert_to_csr(), ([0, 3, 4], [0, 1, 2, 1], np.array([1, 3, 2, 5], NP[dt])))
    # automatic on this 2-row matrix: everything in Coo (csr_kernels.cpp:1301-1309)
    Ha = A.convert_to_hybrid("automatic")
    assert Ha.width == 0 and Ha.coo_row_idxs.cpu().tolist() == [0, 0, 0, 1]


@pytest.mark.parametrize("dt", DTS)
@pytest.mark.parametrize("strategy,kw", [("automatic", {}), ("imbalance_limit", {"percent": 0.5}),
                                         ("imbalance_bounded_limit",
                                          {"percent": 0.9, "ratio": 0.05}),
                                         ("minimal_storage_limit", {}),
                                         ("column_limit", {"num_columns": 3})])
def test_hybrid_random_matches_oracle(exe, dt, strategy, kw):
    rng = np.random.default_rng(11)
    n, m = 20000, 20000
    lens = np.minimum(rng.geometric(0.12, size=n), 200)
    lens[:3] = 0
    rp, ci, v = random_csr(rng, n, m, lens)
    v = v.astype(NP[dt])
    A = dev(exe, (rp, ci, v), (n, m), dt)
    H = A.convert_to_hybrid(strategy, **kw)
    w = S.hybrid_width(lens, strategy, value_bytes=np.dtype(NP[dt]).itemsize, **kw)
    h = S.csr_to_hybrid(rp, ci, v, w)
    assert H.width == w
    np.testing.assert_array_equal(H.ell_col_idxs.cpu().numpy(), h["ell_col_idxs"])
    np.testing.assert_array_equal(H.ell_values.cpu().numpy(), h["ell_values"])
    np.testing.assert_array_equal(H.coo_row_idxs.cpu().numpy(), h["coo_row_idxs"])
    np.testing.assert_array_equal(H.coo_col_idxs.cpu().numpy(), h["coo_col_idxs"])
    np.testing.assert_array_equal(H.coo_values.cpu().numpy(), h["coo_values"])
    # apply: per row the Ell slots then the Coo entries, the oracle's order
    x = rng.standard_normal((m, 3)).astype(NP[dt])
    y = torch.empty((n, 3), dtype=dt, device="cuda")
    H.apply(torch.from_numpy(x).cuda(), y)
    np.testing.assert_array_equal(y.cpu().numpy(), S.hybrid_apply(h, x))
    # advanced apply (alpha A x + beta y) within rounding
    y0 = rng.standard_normal((n, 3)).astype(NP[dt])
    y2 = torch.from_numpy(y0.copy()).cuda()
    H.apply(0.5, torch.from_numpy(x).cuda(), -2.0, y2)
    ref = S.hybrid_apply(h, x.astype(np.float64)) * 0.5 - 2.0 * y0
    tol = 1e-13 if dt == torch.float64 else 1e-5
    scale = np.abs(S.hybrid_apply(dict(h, ell_values=np.abs(h["ell_values"]),
                                       coo_values=np.abs(h["coo_values"])),
                                  np.abs(x).astype(np.float64))) + 2 * np.abs(y0) + 1e-30
    assert (np.abs(y2.cpu().numpy() - ref) / scale).max() <= tol
    # round trip to Csr
    C = H.convert_to_csr()
    assert_same(C, (rp, ci, v))
