"""Adaptive-precision block Jacobi on the GPU
(b2s_jacobi_block_generate_adaptive_*, apply_adaptive, expand, reduce)
against the reference's known answers (tests/golden/jacobi_cases.json,
"adaptive", from reference/test/preconditioner/jacobi_kernels.cpp) and
against the oracle's restatement (oracle.jacobi.generate_adaptive) on seeded
blocks of graded conditioning: the chosen precisions, the conditioning and
the stored blocks bit for bit, the apply within rounding, transposition,
and CG with the adaptive preconditioner."""
import json
import os

import numpy as np
import pytest
import torch

from ginkgo_b200.matrix import Csr, CudaExecutor
from ginkgo_b200.solver import AUTODETECT, BlockJacobi, precision_reduction
from oracle import jacobi as J

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "jacobi_cases.json")) as f:
    G = json.load(f)
DT = [(torch.float64, np.float64), (torch.float32, np.float32)]
ALL = [J.P00, J.P01, J.P02, J.P10, J.P11, J.P20]


@pytest.fixture(scope="module")
def exe():
    return CudaExecutor.create(0)


def _graded_blocks(seed, n_target=400, max_run=8):
    """Csr with runs of rows sharing a pattern (the run plus two far
    columns), each run's diagonal strength and scale drawn over several
    decades, so the blocks' conditioning spans well- to ill-conditioned."""
    rng = np.random.default_rng(seed)
    runs, n = [], 0
    while n < n_target:
        r = int(rng.integers(1, max_run + 1))
        runs.append((n, r))
        n += r
    rows = []
    for s, r in runs:
        pool = np.setdiff1d(np.arange(n), np.arange(max(0, s - 40), s + r + 40))
        far = rng.choice(pool, size=2, replace=False)
        cols = np.unique(np.concatenate([np.arange(s, s + r), far]))
        strength = 10.0 ** rng.uniform(-6, 1.5)
        scale = 10.0 ** rng.uniform(-3, 3)
        for i in range(r):
            vals = rng.uniform(-1, 1, len(cols))
            d = cols == s + i
            vals[d] += strength * r * np.sign(vals[d] + 1e-30)
            rows.append((cols, vals * scale))
    rp = np.concatenate([[0], np.cumsum([len(c) for c, _ in rows])]).astype(np.int32)
    ci = np.concatenate([c for c, _ in rows]).astype(np.int32)
    v = np.concatenate([v for _, v in rows])
    return rp, ci, v


def _check_against_oracle(bj, rp, ci, v, mbs, npdt, accuracy, requests, aggregate_l1=False):
    n = len(rp) - 1
    ref, chosen, conds = J.generate_adaptive(rp, ci, v.astype(npdt), mbs,
                                             block_ptrs=bj.block_pointers, accuracy=accuracy,
                                             precisions=requests, aggregate_l1=aggregate_l1,
                                             dtype=npdt)
    assert bj.block_precisions.tolist() == chosen
    np.testing.assert_array_equal(bj.conditioning.cpu().numpy(), np.array(conds, npdt))
    np.testing.assert_array_equal(bj.to_dense(), J.to_dense(ref, n))
    return ref, chosen


def _requests(case):
    p = case["precisions"]
    return AUTODETECT if p is None else p


@pytest.mark.parametrize("case", G["adaptive"], ids=lambda c: c["name"])
def test_adaptive_known_answers(exe, case):
    # the precisions and conditioning the reference's tests state (FP64)
    m = case["matrix"]
    A = Csr.read(exe, m["row_ptrs"], m["col_idxs"], m["values"], dtype=torch.float64)
    bj = BlockJacobi(A, case["max_block_size"], case["block_ptrs"],
                     storage_optimization=_requests(case), accuracy=case.get("accuracy", 1e-1))
    if "expected" in case:
        assert bj.block_precisions.tolist() == case["expected"]
    if "conditioning" in case:
        np.testing.assert_allclose(bj.conditioning.cpu().numpy(), case["conditioning"],
                                   rtol=1e-14)
    _check_against_oracle(bj, np.array(m["row_ptrs"]), np.array(m["col_idxs"]),
                          np.array(m["values"]), case["max_block_size"], np.float64,
                          case.get("accuracy", 1e-1), case["precisions"])


@pytest.mark.parametrize("case", G["adaptive"], ids=lambda c: c["name"])
def test_adaptive_known_answer_matrices_in_fp32(exe, case):
    m = case["matrix"]
    A = Csr.read(exe, m["row_ptrs"], m["col_idxs"], m["values"], dtype=torch.float32)
    bj = BlockJacobi(A, case["max_block_size"], case["block_ptrs"],
                     storage_optimization=_requests(case), accuracy=case.get("accuracy", 1e-1))
    _check_against_oracle(bj, np.array(m["row_ptrs"]), np.array(m["col_idxs"]),
                          np.array(m["values"]), case["max_block_size"], np.float32,
                          case.get("accuracy", 1e-1), case["precisions"])


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("mbs", [4, 8, 13, 32])
@pytest.mark.parametrize("accuracy", [1e-1, 1e-3])
def test_autodetect_matches_oracle(exe, dt, npdt, mbs, accuracy):
    rp, ci, v = _graded_blocks(mbs * 7 + int(accuracy * 1e4))
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    bj = BlockJacobi(A, mbs, storage_optimization=AUTODETECT, accuracy=accuracy)
    ref, chosen = _check_against_oracle(bj, rp, ci, v, mbs, npdt, accuracy, None)
    if npdt == np.float64 and accuracy == 1e-1:
        assert len(set(chosen)) >= 2  # the graded blocks reach several storages
    # apply, 3 right-hand sides, plain and alpha/beta
    n = len(rp) - 1
    rng = np.random.default_rng(mbs)
    b = rng.standard_normal((n, 3)).astype(npdt)
    x0 = rng.standard_normal((n, 3)).astype(npdt)
    D = J.to_dense(ref, n).astype(np.float64)
    tol = 1e-13 if npdt == np.float64 else 1e-5
    xd = torch.from_numpy(x0.copy()).cuda()
    bj.apply(torch.from_numpy(b).cuda(), xd)
    exp = D @ b.astype(np.float64)
    scale = np.abs(D).sum(axis=1, keepdims=True) * np.abs(b).max() + 1e-300
    assert np.all(np.abs(xd.cpu().numpy() - exp) <= tol * scale)
    xd = torch.from_numpy(x0.copy()).cuda()
    bj.apply(-0.5, torch.from_numpy(b).cuda(), 2.0, xd)
    exp = -0.5 * (D @ b.astype(np.float64)) + 2.0 * x0
    assert np.all(np.abs(xd.cpu().numpy() - exp) <= tol * (scale + np.abs(x0) * 4))


@pytest.mark.parametrize("dt,npdt", DT)
@pytest.mark.parametrize("mbs", [3, 8, 16])
def test_every_storage_type_round_trips(exe, dt, npdt, mbs):
    # each group requests one precision (blocks of a group share it), all
    # six encodings and autodetection in turn; the stored blocks are the
    # full-precision inverses rounded to each storage type
    rp, ci, v = _graded_blocks(100 + mbs)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    probe = BlockJacobi(A, mbs)
    gs = 1 << probe.storage_scheme[2]  # blocks per group
    req = np.repeat(np.array(ALL + [AUTODETECT], np.uint8), gs)
    bj = BlockJacobi(A, mbs, storage_optimization=req)
    nb = bj.num_blocks
    full_req = [int(req[i % len(req)]) for i in range(nb)]
    ref, chosen = _check_against_oracle(bj, rp, ci, v, mbs, npdt, 1e-1, full_req)
    for b in range(nb):
        if full_req[b] != AUTODETECT and (b // gs + 1) * gs <= nb:
            assert chosen[b] == full_req[b]
    # the full-precision blocks rounded to each block's storage
    full = J.generate(rp, ci, v.astype(npdt), mbs, block_ptrs=bj.block_pointers, dtype=npdt)
    for blk, exp, p in zip(ref[2], full[2], chosen):
        np.testing.assert_array_equal(blk, J.storage_roundtrip(exp, p, npdt))
    # transposition keeps each group's storage
    t = bj.transpose()
    assert t.block_precisions.tolist() == chosen
    np.testing.assert_array_equal(t.to_dense(), bj.to_dense().T)
    n = len(rp) - 1
    b = np.random.default_rng(mbs).standard_normal((n, 1)).astype(npdt)
    x = torch.zeros((n, 1), dtype=dt, device="cuda")
    t.apply(torch.from_numpy(b).cuda(), x)
    D = bj.to_dense().T.astype(np.float64)
    tol = 1e-13 if npdt == np.float64 else 1e-5
    # an explicit request skips the feasibility check, so half storage may
    # hold infinities (as the reference's would); rows with them are left out
    ok = np.all(np.isfinite(D), axis=1)
    assert ok.sum() > n // 2
    D = D[ok]
    scale = np.abs(D).sum(axis=1, keepdims=True) * np.abs(b).max() + 1e-300
    assert np.all(np.abs(x.cpu().numpy()[ok] - D @ b.astype(np.float64)) <= tol * scale)


@pytest.mark.parametrize("dt,npdt", DT)
def test_single_precision_for_all_blocks(exe, dt, npdt):
    rp, ci, v = _graded_blocks(5)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    for p in (precision_reduction(0, 1), precision_reduction(1, 0), precision_reduction(2, 0)):
        bj = BlockJacobi(A, 8, storage_optimization=p)
        _check_against_oracle(bj, rp, ci, v, 8, npdt, 1e-1, p)
        assert set(bj.block_precisions.tolist()) == {p}
    # precision_reduction(0, 0) is full precision, no adaptive storage
    assert not BlockJacobi(A, 8, storage_optimization=0).adaptive


@pytest.mark.parametrize("dt,npdt", DT)
def test_adaptive_with_l1(exe, dt, npdt):
    rp, ci, v = _graded_blocks(11)
    A = Csr.read(exe, rp, ci, v, dtype=dt)
    bj = BlockJacobi(A, 8, aggregate_l1=True, storage_optimization=AUTODETECT)
    _check_against_oracle(bj, rp, ci, v, 8, npdt, 1e-1, None, aggregate_l1=True)


def test_cg_with_adaptive_block_jacobi(exe):
    # CG on the 7-point 12^3 operator with 8-row blocks stored adaptively:
    # the fused solver reads each group at its storage precision (widening
    # is exact), so its iterations match the oracle's CG with the oracle's
    # rounded inverses
    from ginkgo_b200 import stencils
    from ginkgo_b200.solver import Cg, Jacobi
    from oracle import oracle as orc
    from test_solvers_gpu import crit
    rp, ci, v = stencils.poisson_3d_7pt(12)
    n = len(rp) - 1
    ptrs = np.concatenate([np.arange(0, n, 8), [n]]).astype(np.int32)
    A = Csr.read(exe, rp, ci, v, dtype=torch.float64)
    s = (Cg.build().with_criteria(*crit(1000, 1e-10))
         .with_preconditioner(Jacobi.build().with_max_block_size(8).with_block_pointers(ptrs)
                              .with_storage_optimization(AUTODETECT))
         .on(exe).generate(A))
    assert s.precond.adaptive
    chosen = s.precond.block_precisions.tolist()
    b = np.random.default_rng(3).standard_normal((n, 1))
    x = torch.zeros((n, 1), dtype=torch.float64, device="cuda")
    s.apply(torch.from_numpy(b).cuda(), x)
    ref, ch_o, _ = J.generate_adaptive(rp, ci, v, 8, block_ptrs=ptrs, precisions=None)
    assert chosen == ch_o and set(chosen) != {J.P00}
    xo, it_o, _, conv_o = orc.cg_block(rp, ci, v, b, ref[1], ref[2], 8, max_iters=1000,
                                       reduction=1e-10)
    assert s.logger.has_converged and conv_o == 1
    assert abs(s.logger.num_iterations - it_o) <= 1
    np.testing.assert_allclose(x.cpu().numpy(), xo.reshape(n, 1), rtol=0,
                               atol=1e-8 * np.abs(xo).max())


def _storage_requests(storage, gs):
    if storage == "f32":
        return J.P01
    if storage == "f16":
        return J.P02
    # groups of different storages: the passes switch per group
    return np.repeat(np.array([J.P01, J.P02, J.P10, J.P20, J.P11, J.P00], np.uint8), gs)


@pytest.mark.parametrize("solver,k", [("cg", 1), ("cg", 4), ("bicgstab", 1), ("gmres", 1)])
@pytest.mark.parametrize("storage", ["f32", "f16", "mixed"])
def test_solvers_with_adaptive_blocks(exe, solver, k, storage):
    # every group FP32 or every group FP16 (the one-column passes then run an
    # instance fixed to that storage) or groups of different storages (the
    # per-group switch), 8-row blocks, FP64; each solver against the
    # oracle's solver with the oracle's rounded blocks
    from ginkgo_b200 import stencils
    from ginkgo_b200.solver import Bicgstab, Cg, Gmres, Jacobi
    from oracle import oracle as orc
    from test_solvers_gpu import _aniso, crit, explicit_rel_res
    if solver == "cg":
        rp, ci, v = stencils.poisson_3d_7pt(12)
    elif solver == "bicgstab":
        rp, ci, v = stencils.convection_diffusion_2d(40, 36, 1.0, 0.7, -0.4)
    else:
        rp, ci, v, _, _ = _aniso(12)
    n = len(rp) - 1
    mbs = 8
    ptrs = np.concatenate([np.arange(0, n, mbs), [n]]).astype(np.int32)
    req = _storage_requests(storage, 4)  # 4 blocks of 8 rows per group
    b = np.random.default_rng(k + len(storage)).standard_normal((n, k))
    A = Csr.read(exe, rp, ci, v, dtype=torch.float64)
    jac = (Jacobi.build().with_max_block_size(mbs).with_block_pointers(ptrs)
           .with_storage_optimization(req))
    f = {"cg": Cg.build(), "bicgstab": Bicgstab.build(),
         "gmres": Gmres.build().with_krylov_dim(30).with_ortho_method("cgs2")}[solver]
    s = f.with_criteria(*crit(3000, 1e-10)).with_preconditioner(jac).on(exe).generate(A)
    assert s.precond.adaptive
    chosen = s.precond.block_precisions
    if storage == "mixed":
        assert len(set(chosen.tolist())) >= 5
    else:
        assert set(chosen.tolist()) == {int(req)}
    x = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    s.apply(torch.from_numpy(b).cuda(), x)
    assert s.logger.has_converged
    xg = x.cpu().numpy()
    assert np.all(explicit_rel_res(rp, ci, v, xg, b) <= 2e-10)
    ref, ch_o, _ = J.generate_adaptive(rp, ci, v, mbs, block_ptrs=ptrs,
                                       precisions=req if np.isscalar(req) else
                                       [int(req[i % len(req)]) for i in range(len(ptrs) - 1)])
    assert chosen.tolist() == ch_o
    its = []
    for j in range(k):
        if solver == "cg":
            xo, it_o, _, conv = orc.cg_block(rp, ci, v, b[:, j].copy(), ref[1], ref[2], mbs,
                                             max_iters=3000, reduction=1e-10)
        elif solver == "bicgstab":
            xo, it_o, _, conv = orc.bicgstab_block(rp, ci, v, b[:, j].copy(), ref[1], ref[2],
                                                   mbs, max_iters=3000, reduction=1e-10)
        else:
            xo, it_o, _, conv = orc.gmres_block(rp, ci, v, b[:, j].copy(), ref[1], ref[2], mbs,
                                                krylov_dim=30, max_iters=3000,
                                                reduction=1e-10, ortho="cgs2")
        assert conv
        its.append(it_o)
        xo = np.asarray(xo).reshape(-1)
        np.testing.assert_allclose(xg[:, j], xo, rtol=0, atol=1e-7 * np.abs(xo).max())
    slack = {"cg": 1, "bicgstab": max(3, 0.05 * max(its)), "gmres": max(2, 0.01 * max(its))}
    assert abs(s.logger.num_iterations - max(its)) <= slack[solver], \
        (s.logger.num_iterations, its)
