"""Block Jacobi on the GPU (b2s_jacobi_block_generate/apply) against the
reference's known answers (tests/golden/jacobi_cases.json, from
reference/test/preconditioner/jacobi_kernels.cpp) and against the oracle's
restatement on seeded random block patterns, pivoting and singular blocks
included."""
import json
import os

import numpy as np
import pytest
import torch

from ginkgo_b200.matrix import Csr, CudaExecutor
from ginkgo_b200.solver import BlockJacobi, Jacobi
from oracle import jacobi as J

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "jacobi_cases.json")) as f:
    G = json.load(f)
DT = [(torch.float64, np.float64), (torch.float32, np.float32)]


@pytest.fixture(scope="module")
def exe():
    return CudaExecutor.create(0)


def _csr(exe, m, dt):
    return Csr.read(exe, m["row_ptrs"], m["col_idxs"], m["values"], dtype=dt)


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("case", G["dense"], ids=lambda c: c["name"])
def test_inverted_blocks_known_answers(exe, case, dt, npdt):
    A = _csr(exe, case["matrix"], dt)
    bj = BlockJacobi(A, case["max_block_size"], case.get("block_ptrs"),
                     aggregate_l1=case.get("aggregate_l1", False))
    if case.get("transpose"):
        bj = bj.transpose()
    got = bj.to_dense()
    assert np.abs(got - np.array(case["expected"])).max() <= 10 * np.finfo(npdt).eps


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("case", G["apply"], ids=lambda c: c["name"])
def test_apply_known_answers(exe, case, dt, npdt):
    A = _csr(exe, G["dense"][0]["matrix"], dt)
    if case["max_block_size"] == 1:
        p = Jacobi(A)
    else:
        p = BlockJacobi(A, case["max_block_size"], case.get("block_ptrs"))
    b = torch.tensor(case["b"], dtype=dt, device="cuda")
    x = torch.tensor(case["x"], dtype=dt, device="cuda")
    if "alpha" in case:
        p.apply(case["alpha"], b, case["beta"], x)
    else:
        p.apply(b, x)
    got, exp = x.cpu().double().numpy(), np.array(case["expected"])
    err = np.linalg.norm(got - exp) / max(np.linalg.norm(got), np.linalg.norm(exp))
    assert err <= 10 * np.finfo(npdt).eps, (case["name"], err)


def _random_blocks(seed, n_target=600, max_run=9, pivoting=False, singular=False):
    """Csr with runs of rows sharing a pattern: each run's columns are the
    run itself plus a few far columns; diagonally dominant values, or (with
    pivoting) zero diagonals in some runs; one run singular when asked."""
    rng = np.random.default_rng(seed)
    if pivoting:
        max_run = 4  # a run never straddles blocks of 4 or more rows
    runs, n = [], 0
    while n < n_target:
        r = int(rng.integers(1, max_run + 1))
        runs.append((n, r))
        n += r
    rows = []
    for k, (s, r) in enumerate(runs):
        # far columns at least 40 rows away, so they never fall inside a
        # (merged) block: every block stays block-diagonal in its runs
        pool = np.setdiff1d(np.arange(n), np.arange(max(0, s - 40), s + r + 40))
        far = rng.choice(pool, size=3, replace=False)
        cols = np.unique(np.concatenate([np.arange(s, s + r), far]))
        for i in range(r):
            vals = rng.uniform(-1, 1, len(cols))
            row = s + i
            if pivoting and k % 3 == 0:
                # zero diagonal, the strong entry one column to the right
                # (cyclically): every elimination step must swap rows
                vals[cols == row] = 0.0
                vals[cols == s + (i + 1) % r] = 2.0 * r + 4.0
            else:
                vals[cols == row] = 2.0 * r + 4.0
            if singular and k == 1:
                vals[cols == s] = 0.0  # first column of the block is all zero
            rows.append((cols, vals))
    rp = np.concatenate([[0], np.cumsum([len(c) for c, _ in rows])]).astype(np.int32)
    ci = np.concatenate([c for c, _ in rows]).astype(np.int32)
    v = np.concatenate([v for _, v in rows])
    return rp, ci, v


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("mbs", [4, 13, 32])
@pytest.mark.parametrize("kind", ["dominant", "pivoting", "singular"])
def test_random_blocks_match_oracle(exe, dt, npdt, mbs, kind):
    rp, ci, v = _random_blocks(mbs * 10 + len(kind), pivoting=kind == "pivoting",
                               singular=kind == "singular")
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    bj = BlockJacobi(A, mbs)
    assert bj.block_pointers.tolist() == J.find_blocks(rp, ci, mbs)
    ref = J.generate(rp, ci, v.astype(npdt), mbs, dtype=npdt)
    got = bj.to_dense()
    exp = J.to_dense(ref, n)
    tol = 1e-11 if npdt == np.float64 else 2e-4
    scale = max(1.0, np.abs(exp).max())
    assert np.abs(got - exp).max() <= tol * scale
    # apply, 3 right-hand sides, plain and alpha/beta
    rng = np.random.default_rng(mbs)
    b = rng.standard_normal((n, 3)).astype(npdt)
    x0 = rng.standard_normal((n, 3)).astype(npdt)
    bd = torch.from_numpy(b).cuda()
    xd = torch.from_numpy(x0.copy()).cuda()
    bj.apply(bd, xd)
    np.testing.assert_allclose(xd.cpu().numpy(), J.apply(ref, b), rtol=0,
                               atol=tol * scale * np.abs(b).max() * 40)
    xd = torch.from_numpy(x0.copy()).cuda()
    bj.apply(-0.5, bd, 2.0, xd)
    np.testing.assert_allclose(xd.cpu().numpy(), J.apply(ref, b, x0, -0.5, 2.0), rtol=0,
                               atol=tol * scale * np.abs(b).max() * 40 + tol * 4)


@pytest.mark.parametrize("mbs,scheme", [(3, (3, 72, 3)), (8, (8, 256, 2)), (13, (13, 338, 1)),
                                        (32, (32, 1024, 0))])
def test_blocks_use_the_reference_interleaved_layout(exe, mbs, scheme):
    """The raw blocks array is the reference's block_interleaved_storage_scheme
    (jacobi.hpp:589-621 with the CUDA block stride of 32): group size
    32 / pow2ceil(max_block_size), block_offset = max_block_size,
    stride = group size * block_offset, group_offset = max_block_size * stride;
    entry (i, j) of block b at get_global_block_offset(b) + i + j * stride."""
    rp, ci, v = _random_blocks(mbs + 100)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    bj = BlockJacobi(A, mbs)
    assert bj.storage_scheme == scheme
    bo, go, gp = scheme
    gs = 1 << gp
    stride = bo << gp
    nb = bj.num_blocks
    assert bj.blocks.numel() == -(-nb // gs) * go  # compute_storage_space
    raw = bj.blocks.cpu().numpy()
    ref = J.to_dense(J.generate(rp, ci, v, mbs), n)
    ptrs = bj.block_pointers
    for b in range(nb):
        s, e = ptrs[b], ptrs[b + 1]
        off = go * (b >> gp) + bo * (b & (gs - 1))
        for i in range(e - s):
            for j in range(e - s):
                assert abs(raw[off + i + j * stride] - ref[s + i, s + j]) <= \
                    1e-11 * max(1.0, abs(ref[s + i, s + j])), (b, i, j)


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("case", G["l1"], ids=lambda c: c["name"])
def test_l1_known_answers(exe, case, dt, npdt):
    # aggregate_l1 on the device: the scalar case's modified diagonal (as
    # its inverse) and the block case's modified blocks (as their inverses)
    m = case["matrix"]
    A = _csr(exe, m, dt)
    if case["kind"] == "scalar":
        got = Jacobi(A, aggregate_l1=True).inv_diag.cpu().numpy()
        exp = 1.0 / np.array(case["expected"], npdt)
        np.testing.assert_array_equal(got, exp)
    else:
        ptrs = case["block_ptrs"]
        bj = BlockJacobi(A, max(np.diff(ptrs)), ptrs, aggregate_l1=True)
        d = np.array(case["expected"], np.float64)
        exp = np.zeros_like(d)
        for s0, e0 in zip(ptrs[:-1], ptrs[1:]):
            exp[s0:e0, s0:e0] = J.invert_block(d[s0:e0, s0:e0].astype(npdt))
        assert np.abs(bj.to_dense() - exp).max() <= 10 * np.finfo(npdt).eps


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("mbs", [1, 4, 13])
def test_l1_random_blocks_match_oracle(exe, dt, npdt, mbs):
    # aggregate_l1 with rows reaching outside their blocks: the 27-point
    # 8^3 operator in uniform blocks of mbs rows, against the oracle
    from ginkgo_b200 import stencils
    rp, ci, v = stencils.anisotropic_27pt(8)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    ptrs = np.concatenate([np.arange(0, n, mbs), [n]]).astype(np.int32)
    if mbs == 1:
        got = Jacobi(A, aggregate_l1=True).inv_diag.cpu().numpy()
        _, exp = J.generate(rp, ci, v.astype(npdt), 1, aggregate_l1=True, dtype=npdt)
        np.testing.assert_array_equal(got, exp)
        return
    bj = BlockJacobi(A, mbs, ptrs, aggregate_l1=True)
    ref = J.generate(rp, ci, v.astype(npdt), mbs, block_ptrs=ptrs, aggregate_l1=True,
                     dtype=npdt)
    exp = J.to_dense(ref, n)
    tol = 1e-12 if npdt == np.float64 else 2e-5
    assert np.abs(bj.to_dense() - exp).max() <= tol * max(1.0, np.abs(exp).max())
