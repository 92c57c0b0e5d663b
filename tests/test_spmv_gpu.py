"""SpMV and format conversion on the GPU against the CPU oracle.

Tolerances: FP64 results agree with the oracle to 1e-14 relative, scaled by
the row's absolute sum |A||x| (the reduction order differs); FP32 to 1e-5 on
the same scale.  Conversions, row pointers and patterns are bit-exact.
"""
import numpy as np
import pytest
import torch

from conftest import dense_to_csr, to_array
from ginkgo_b200 import stencils
from ginkgo_b200.matrix import Csr, CudaExecutor
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-14, torch.float32: 1e-5}
NP = {torch.float64: np.float64, torch.float32: np.float32}


@pytest.fixture(scope="module")
def exe():
    return CudaExecutor.create(0)


def assert_spmv_close(rp, ci, v, x, got, ref, tol, alpha=1.0, beta_y=None):
    """|got - ref| <= tol * (|alpha| |A| |x| + |beta y|) row by row."""
    absA = np.abs(v).astype(np.float64)
    scale = abs(alpha) * orc.csr_spmv(rp, ci, absA, np.abs(x).astype(np.float64))
    if beta_y is not None:
        scale = scale + np.abs(beta_y).reshape(scale.shape)
    scale = np.maximum(scale, np.finfo(np.float64).tiny)
    err = np.abs(got.astype(np.float64) - ref.astype(np.float64)) / scale
    assert err.max() <= tol, err.max()


def formats(A, fmt):
    if fmt == "classical":
        return A.set_strategy("classical")
    if fmt == "load_balance":
        return A.set_strategy("load_balance")
    if fmt == "ell":
        return A.convert_to_ell()
    if fmt == "sellp":
        return A.convert_to_sellp(32, 1)
    raise ValueError(fmt)


FORMATS = ["classical", "load_balance", "ell", "sellp"]


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_known_answers(exe, known, fmt, dt):
    for case in known["spmv"]:
        m = case["matrix"]
        A = Csr(exe, (m["n_rows"], m["n_cols"]), m["row_ptrs"], m["col_idxs"],
                torch.tensor(m["values"], dtype=dt))
        op = formats(A, fmt)
        x = torch.tensor(to_array(case["x"]), dtype=dt, device="cuda")
        if "alpha" in case:
            y = torch.tensor(to_array(case["y"]), dtype=dt, device="cuda")
            op.apply(case["alpha"], x, case["beta"], y)
        else:
            y = torch.empty((2, x.shape[1]), dtype=dt, device="cuda")
            op.apply(x, y)
        np.testing.assert_array_equal(y.cpu().numpy(),
                                      to_array(case["expected"], NP[dt]),
                                      err_msg=f"{fmt} {case['name']}")


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("k", [1, 3, 4, 16])
def test_random_power_law_matches_oracle(exe, fmt, dt, k):
    # long rows (up to 3000 > the 2048-entry chunk), empty-free, unsorted
    rng = np.random.default_rng(7 + k)
    rp, ci, v = stencils.power_law(20000, seed=11, mu=2.0, sigma=1.2, max_len=3000)
    v = v.astype(NP[dt])
    x = rng.standard_normal((20000, k)).astype(NP[dt])
    ref = orc.csr_spmv(rp, ci, v, x)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    op = formats(A, fmt)
    xd = torch.from_numpy(x).cuda()
    y = torch.full((20000, k), float("nan"), dtype=dt, device="cuda")
    op.apply(xd, y)
    assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, TOL[dt])
    # advanced apply, beta != 0
    y0 = rng.standard_normal((20000, k)).astype(NP[dt])
    ref2 = orc.csr_spmv(rp, ci, v, x, y0, -0.5, 2.0)
    y2 = torch.from_numpy(y0).cuda()
    op.apply(-0.5, xd, 2.0, y2)
    assert_spmv_close(rp, ci, v, x, y2.cpu().numpy(), ref2, TOL[dt] * 4,
                      alpha=0.5, beta_y=2.0 * y0.astype(np.float64))


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("k", [1, 2])
def test_classical_every_group_width(exe, dt, k):
    # The pipelined kernel groups 32 / lpr rows per warp (lpr 1, 2 or 4),
    # chosen from the longest row; the row-length bound handed to it only
    # changes the grouping, so every width (and groups that overflow a
    # stage) must give the same result.  Rows of 0..60 entries, a few of 400.
    rng = np.random.default_rng(21 + k)
    n = 30001
    lens = rng.integers(0, 61, n)
    lens[rng.choice(n, 20, replace=False)] = 400
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([rng.choice(n, l, replace=False) for l in lens]).astype(np.int32)
    v = rng.standard_normal(int(rp[-1])).astype(NP[dt])
    x = rng.standard_normal((n, k)).astype(NP[dt])
    ref = orc.csr_spmv(rp, ci, v, x)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    xd = torch.from_numpy(x).cuda()
    for bound in (1, 8, 16, 32, 64, 128, 256, 400):
        A._max_row_nnz = bound
        y = torch.full((n, k), float("nan"), dtype=dt, device="cuda")
        A.apply(xd, y)
        assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, TOL[dt])


@pytest.mark.parametrize("fmt", ["classical", "load_balance"])
def test_empty_rows_and_single_long_row(exe, fmt):
    n = 9000
    lens = np.zeros(n, np.int64)
    lens[::3] = 2          # every third row has two entries, the rest empty
    lens[4500] = 7000      # one row spanning several load_balance chunks
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    rng = np.random.default_rng(5)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    v = rng.standard_normal(int(rp[-1]))
    x = rng.standard_normal((n, 2))
    ref = orc.csr_spmv(rp, ci, v, x)
    A = formats(Csr.read(exe, rp, ci, v), fmt)
    y = torch.full((n, 2), float("nan"), dtype=torch.float64, device="cuda")
    A.apply(torch.from_numpy(x).cuda(), y)
    assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, 1e-14)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("k", [1, 5, 20])
def test_load_balance_chunk_boundaries(exe, dt, k):
    # load_balance cuts the entries into 256-entry chunks: rows that end
    # exactly on a boundary, rows of 250..260 entries that straddle one or
    # two, runs of empty rows at boundaries and at the end, rows longer than a
    # warp inside a chunk, and nnz a multiple of 256.  k = 20 runs two column
    # passes (16 + 4) over the same partial-sum scratch; plain and advanced.
    rng = np.random.default_rng(31 + k)
    n = 6000
    lens = rng.choice([0, 0, 0, 1, 3, 40, 250, 256, 260, 600], n)
    lens[-50:] = 0
    lens[0] = 256
    total = int(lens.sum())
    lens[1] += (-total) % 256  # nnz a multiple of 256
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([rng.choice(n, l, replace=False) for l in lens]).astype(np.int32)
    v = rng.standard_normal(int(rp[-1])).astype(NP[dt])
    x = rng.standard_normal((n, k)).astype(NP[dt])
    y0 = rng.standard_normal((n, k)).astype(NP[dt])
    A = Csr.read(exe, rp, ci, v, dtype=dt).set_strategy("load_balance")
    xd = torch.from_numpy(x).cuda()
    y = torch.full((n, k), float("nan"), dtype=dt, device="cuda")
    A.apply(xd, y)
    assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), orc.csr_spmv(rp, ci, v, x), TOL[dt])
    y2 = torch.from_numpy(y0).cuda()
    A.apply(0.75, xd, -2.0, y2)
    assert_spmv_close(rp, ci, v, x, y2.cpu().numpy(), orc.csr_spmv(rp, ci, v, x, y0, 0.75, -2.0),
                      TOL[dt] * 4, alpha=0.75, beta_y=2.0 * y0.astype(np.float64))
    # run to run identical: no atomics in the partial sums
    y3 = torch.full((n, k), float("nan"), dtype=dt, device="cuda")
    A.apply(xd, y3)
    assert torch.equal(y, y3)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("k", [4, 8, 16])
def test_ell_sellp_row_pairs_many_rhs(exe, dt, k):
    # four or more right-hand sides on Ell / Sellp: row pairs per lane slot
    # when the stride (Ell) or slice size (Sellp) is even, single rows when
    # it is odd; an odd row count leaves the last pair half inside the
    # matrix (with Ell stride n + 1 its second row is padding storage)
    rng = np.random.default_rng(60 + k)
    n = 4097
    lens = rng.integers(0, 12, n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    v = rng.standard_normal(int(rp[-1])).astype(NP[dt])
    x = rng.standard_normal((n, k)).astype(NP[dt])
    y0 = rng.standard_normal((n, k)).astype(NP[dt])
    ref = orc.csr_spmv(rp, ci, v, x)
    ref2 = orc.csr_spmv(rp, ci, v, x, y0, 0.5, -2.0)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    ops = [A.convert_to_ell(stride=n), A.convert_to_ell(stride=n + 1)]
    ops += [A.convert_to_sellp(ss, 1) for ss in (2, 7, 32)]
    xd = torch.from_numpy(x).cuda()
    for op in ops:
        y = torch.full((n, k), float("nan"), dtype=dt, device="cuda")
        op.apply(xd, y)
        assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, TOL[dt])
        y2 = torch.from_numpy(y0).cuda()
        op.apply(0.5, xd, -2.0, y2)
        assert_spmv_close(rp, ci, v, x, y2.cpu().numpy(), ref2, TOL[dt] * 4,
                          alpha=0.5, beta_y=2.0 * y0.astype(np.float64))
    # Sellp through the plain entry point (no longest-slice hint: one row
    # per lane slot) and through the hinted one with a hint that rules pairs
    # out (a slice longer than the pairing bound): the same products
    from ginkgo_b200._lib import call
    from ginkgo_b200.matrix import _p, _stream
    sfx = "f64" if dt == torch.float64 else "f32"
    S = A.convert_to_sellp(32, 1)
    assert 0 < S.max_slice_length <= 12
    for entry, hint in ((f"b2s_sellp_spmv_{sfx}", None), (f"b2s_sellp_spmv_hinted_{sfx}", 100)):
        y = torch.full((n, k), float("nan"), dtype=dt, device="cuda")
        args = [n, n, 32, _p(S.slice_sets), _p(S.slice_lengths), _p(S.col_idxs), _p(S.values),
                _p(xd), xd.stride(0), _p(y), y.stride(0), k, None, None]
        if hint is not None:
            args.append(hint)
        call(entry, *args, _stream(y))
        assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, TOL[dt])


@pytest.mark.parametrize("fmt", FORMATS)
def test_empty_matrix(exe, fmt):
    A = Csr(exe, (0, 0), torch.zeros(1, dtype=torch.int32), torch.zeros(0, dtype=torch.int32),
            torch.zeros(0, dtype=torch.float64))
    op = formats(A, fmt)
    x = torch.zeros((0, 1), dtype=torch.float64, device="cuda")
    y = torch.zeros((0, 1), dtype=torch.float64, device="cuda")
    op.apply(x, y)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_ell_sellp_one_rhs_row_groups(exe, dt):
    # one right-hand side runs R = 16 / sizeof(value) rows per thread when
    # the layout allows 16-byte loads, the row-per-thread kernel otherwise;
    # all against the oracle, plain and advanced
    rp, ci, v = stencils.anisotropic_27pt(15)
    n = len(rp) - 1
    v = v.astype(NP[dt])
    rng = np.random.default_rng(9)
    x = rng.standard_normal((n, 1)).astype(NP[dt])
    y0 = rng.standard_normal((n, 1)).astype(NP[dt])
    ref = orc.csr_spmv(rp, ci, v, x)
    ref2 = orc.csr_spmv(rp, ci, v, x, y0, 0.5, -1.5)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    # Ell with an odd and an even stride; Sellp with a slice size that is
    # not a multiple of the row group (7) and two that are (32, 64; the last
    # slice partial)
    ops = [A.convert_to_ell(stride=n), A.convert_to_ell(stride=n + 1)]
    ops += [A.convert_to_sellp(ss, sf) for ss, sf in ((7, 1), (32, 1), (64, 2))]
    for E in ops:
        y = torch.full((n, 1), float("nan"), dtype=dt, device="cuda")
        E.apply(torch.from_numpy(x).cuda(), y)
        assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, TOL[dt])
        y2 = torch.from_numpy(y0).cuda()
        E.apply(0.5, torch.from_numpy(x).cuda(), -1.5, y2)
        assert_spmv_close(rp, ci, v, x, y2.cpu().numpy(), ref2, TOL[dt] * 4,
                          alpha=0.5, beta_y=1.5 * y0.astype(np.float64))


def test_conversions_bit_exact(exe, known):
    rp, ci, v = stencils.power_law(5000, seed=2, mu=1.8, max_len=400)
    A = Csr.read(exe, rp, ci, v)
    w, s, eci, ev = orc.csr_to_ell(rp, ci, v)
    E = A.convert_to_ell()
    assert (E.width, E.stride) == (w, s)
    np.testing.assert_array_equal(E.col_idxs.cpu().numpy(), eci)
    np.testing.assert_array_equal(E.values.cpu().numpy(), ev)
    for ss, sf in [(32, 1), (64, 1), (2, 2), (7, 3)]:
        sets, lens, sci, sv = orc.csr_to_sellp(rp, ci, v, ss, sf)
        S = A.convert_to_sellp(ss, sf)
        np.testing.assert_array_equal(S.slice_sets.cpu().numpy(), sets.astype(np.int64))
        np.testing.assert_array_equal(S.slice_lengths.cpu().numpy(), lens.astype(np.int64))
        np.testing.assert_array_equal(S.col_idxs.cpu().numpy(), sci)
        np.testing.assert_array_equal(S.values.cpu().numpy(), sv)
    case = known["convert_to_sellp"]
    m = case["matrix"]
    S = Csr(exe, (2, 3), m["row_ptrs"], m["col_idxs"],
            torch.tensor(m["values"], dtype=torch.float64)).convert_to_sellp(64, 1)
    np.testing.assert_array_equal(S.slice_sets.cpu().numpy(), case["slice_sets"])
    for idx, (c, val) in case["checks"].items():
        assert S.col_idxs[int(idx)].item() == c and S.values[int(idx)].item() == val


def test_transpose_bit_exact(exe, known):
    for case in known["transpose"]:
        d = np.array(case["dense"])
        rp, ci, v = dense_to_csr(d)
        T = Csr.read(exe, rp, ci, v, shape=d.shape).transpose()
        erp, eci, ev = dense_to_csr(case["expected_dense"])
        np.testing.assert_array_equal(T.row_ptrs.cpu().numpy(), erp)
        np.testing.assert_array_equal(T.col_idxs.cpu().numpy(), eci)
        np.testing.assert_array_equal(T.values.cpu().numpy(), ev)
    rp, ci, v = stencils.power_law(6000, seed=4, mu=2.0, max_len=300)
    trp, tci, tv = orc.csr_transpose(rp, ci, v, 6000)
    T = Csr.read(exe, rp, ci, v).transpose()
    np.testing.assert_array_equal(T.row_ptrs.cpu().numpy(), trp)
    np.testing.assert_array_equal(T.col_idxs.cpu().numpy(), tci)
    np.testing.assert_array_equal(T.values.cpu().numpy(), tv)


def test_poisson_128_full_size_fp64(exe):
    """The benchmark matrix (3D 7-point, 128^3) at full size, k = 1 and 16."""
    rp, ci, v = stencils.poisson_3d_7pt(128)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    rng = np.random.default_rng(0)
    for k in (1, 16):
        x = rng.standard_normal((n, k))
        ref = orc.csr_spmv(rp, ci, v, x)
        xd = torch.from_numpy(x).cuda()
        for fmt in FORMATS:
            op = formats(A, fmt)
            y = torch.empty((n, k), dtype=torch.float64, device="cuda")
            op.apply(xd, y)
            assert_spmv_close(rp, ci, v, x, y.cpu().numpy(), ref, 1e-14)


MIXED = [(m, i, o) for m in (torch.float64, torch.float32)
         for i in (torch.float64, torch.float32) for o in (torch.float64, torch.float32)]


def _mixed_tol(m, i, o):
    # arithmetic in the most precise type; one rounding to the output type
    if o == torch.float64:
        return 1e-14  # FP64 arithmetic, FP64 result
    return 1e-6 if torch.float64 in (m, i) else 1e-5


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("m,i,o", MIXED, ids=lambda t: str(t).split(".")[-1])
@pytest.mark.parametrize("k", [1, 3, 20])
def test_mixed_value_types_match_oracle(exe, fmt, m, i, o, k):
    """Matrix, b and x each FP64 or FP32 (Csr and Ell compute in the most
    precise type; Sellp converts the operands to its own type)."""
    rng = np.random.default_rng(31 + k)
    rp, ci, v = stencils.power_law(6000, seed=13, mu=2.0, sigma=1.0, max_len=600)
    n = len(rp) - 1
    vm = v.astype(NP[m])
    x = rng.standard_normal((n, k)).astype(NP[i])
    y0 = rng.standard_normal((n, k)).astype(NP[o])
    A = Csr.read(exe, rp, ci, vm, dtype=m)
    op = formats(A, fmt)
    # what the operator computes from: Sellp rounds b and x to its own type
    xs = x.astype(NP[m]) if fmt == "sellp" else x
    ref = orc.csr_spmv(rp, ci, vm.astype(np.float64), xs.astype(np.float64))
    tol = _mixed_tol(m, i, o)
    if fmt == "sellp":
        tol = TOL[m] if o == torch.float64 or m == torch.float32 else 1e-6
    y = torch.full((n, k), float("nan"), dtype=o, device="cuda")
    op.apply(torch.from_numpy(x).cuda(), y)
    assert_spmv_close(rp, ci, vm, xs, y.cpu().numpy(), ref, max(tol, 1e-14))
    # advanced: alpha in the matrix type, beta in the output type
    y0s = y0.astype(NP[m]) if fmt == "sellp" else y0
    ref2 = 0.75 * ref - 1.25 * y0s.astype(np.float64)
    y2 = torch.from_numpy(y0.copy()).cuda()
    op.apply(0.75, torch.from_numpy(x).cuda(), -1.25, y2)
    assert_spmv_close(rp, ci, vm, xs, y2.cpu().numpy(), ref2, max(tol, 1e-14) * 4,
                      alpha=0.75, beta_y=1.25 * y0s.astype(np.float64))


def test_dense_convert_round_trip(exe):
    from ginkgo_b200.matrix import _convert
    x = torch.randn(1000, 5, dtype=torch.float64, device="cuda")[:, :3]
    f = _convert(x, torch.float32)
    assert f.dtype == torch.float32 and torch.equal(f, x.float())
    d = _convert(f, torch.float64)
    assert torch.equal(d, x.float().double())
