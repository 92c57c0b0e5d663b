"""Pins the CPU oracle to the reference's known answers (no GPU needed)."""
import numpy as np
import pytest

from conftest import dense_to_csr, std_uniform, to_array
from ginkgo_b200 import stencils
from oracle import oracle as orc

DTYPES = [np.float64, np.float32]


def _mtx(case, dt):
    m = case["matrix"]
    return (np.array(m["row_ptrs"], np.int32), np.array(m["col_idxs"], np.int32),
            np.array(m["values"], dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_spmv_known_answers(known, dt):
    for case in known["spmv"]:
        rp, ci, v = _mtx(case, dt)
        x = to_array(case["x"], dt)
        if "alpha" in case:
            y = orc.csr_spmv(rp, ci, v, x, to_array(case["y"], dt),
                             case["alpha"], case["beta"])
        else:
            y = orc.csr_spmv(rp, ci, v, x)
        np.testing.assert_array_equal(y, to_array(case["expected"], dt),
                                      err_msg=case["name"])


@pytest.mark.parametrize("dt", DTYPES)
def test_convert_to_ell_known_answer(known, dt):
    case = known["convert_to_ell"]
    rp, ci, v = _mtx(case, dt)
    w, s, eci, ev = orc.csr_to_ell(rp, ci, v)
    assert (w, s) == (case["width"], case["stride"])
    np.testing.assert_array_equal(eci, case["col_idxs"])
    np.testing.assert_array_equal(ev, np.array(case["values"], dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_convert_to_sellp_known_answer(known, dt):
    case = known["convert_to_sellp"]
    rp, ci, v = _mtx(case, dt)
    sets, lens, sci, sv = orc.csr_to_sellp(rp, ci, v, case["slice_size"],
                                           case["stride_factor"])
    np.testing.assert_array_equal(sets, case["slice_sets"])
    np.testing.assert_array_equal(lens, case["slice_lengths"])
    for idx, (c, val) in case["checks"].items():
        assert sci[int(idx)] == c and sv[int(idx)] == val


@pytest.mark.parametrize("dt", DTYPES)
def test_sellp_slice_size_stride_factor(known, dt):
    case = known["sellp_slice2_stride2"]
    rp, ci, v = _mtx(case, dt)
    sets, lens, sci, sv = orc.csr_to_sellp(rp, ci, v, case["slice_size"],
                                           case["stride_factor"])
    x = to_array(case["x"], dt)
    y = orc.sellp_spmv(2, case["slice_size"], sets, lens, sci, sv, x)
    np.testing.assert_array_equal(y, to_array(case["expected_simple"], dt))
    y = orc.sellp_spmv(2, case["slice_size"], sets, lens, sci, sv, x,
                       to_array(case["y"], dt), case["alpha"], case["beta"])
    np.testing.assert_array_equal(y, to_array(case["expected_advanced"], dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_ell_with_stride(known, dt):
    case = known["ell_stride16"]
    rp, ci, v = _mtx(case, dt)
    w, s, eci, ev = orc.csr_to_ell(rp, ci, v, stride=case["stride"])
    y = orc.ell_spmv(2, w, s, eci, ev, to_array(case["x"], dt))
    np.testing.assert_array_equal(y, to_array(case["expected"], dt))


def test_transpose_known_answers(known):
    for case in known["transpose"]:
        d = np.array(case["dense"])
        rp, ci, v = dense_to_csr(d)
        trp, tci, tv = orc.csr_transpose(rp, ci, v, d.shape[1])
        erp, eci, ev = dense_to_csr(case["expected_dense"])
        np.testing.assert_array_equal(trp, erp)
        np.testing.assert_array_equal(tci, eci)
        np.testing.assert_array_equal(tv, ev)


@pytest.mark.parametrize("dt", DTYPES)
def test_cg_step_kernels(known, dt):
    kc = known["cg_kernels"]
    for key in ("step_1", "step_1_div_by_zero"):
        c = kc[key]
        p = np.full((2, 2), c["p"], dt)
        orc.cg_step_1(p, np.full((2, 2), c["z"], dt), c["rho"], c["prev_rho"],
                      c["stopped"])
        np.testing.assert_array_equal(p, np.array(c["expected_p"], dt))
    for key in ("step_2", "step_2_div_by_zero"):
        c = kc[key]
        x = np.full((2, 2), c["x"], dt)
        r = np.full((2, 2), c["r"], dt)
        orc.cg_step_2(x, r, np.full((2, 2), c["p"], dt),
                      np.full((2, 2), c["q"], dt), c["beta"], c["rho"],
                      c["stopped"])
        np.testing.assert_array_equal(x, np.array(c["expected_x"], dt))
        np.testing.assert_array_equal(r, np.array(c["expected_r"], dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_gmres_hessenberg_qr(known, dt):
    eps = np.finfo(dt).eps * 10
    for key in ("hessenberg_qr_iter0", "hessenberg_qr_iter1"):
        c = known["gmres_kernels"][key]
        gs, gc = to_array(c["givens_sin"], dt), to_array(c["givens_cos"], dt)
        rnc = to_array(c["residual_norm_collection"], dt)
        h = to_array(c["hessenberg_iter"], dt)
        rn = np.full(2, np.nan, dt)
        fin = np.full(2, c["iteration"], np.int64)
        orc.gmres_hessenberg_qr(c["iteration"], gs, gc, rn, rnc, h, fin, [0, 0])
        assert list(fin) == [c["iteration"] + 1] * 2
        np.testing.assert_allclose(gc, c["expected_givens_cos"], rtol=eps, atol=eps)
        np.testing.assert_allclose(gs, c["expected_givens_sin"], rtol=eps, atol=eps)
        np.testing.assert_allclose(h, c["expected_hessenberg_iter"], rtol=eps, atol=eps)
        np.testing.assert_allclose(rnc, c["expected_residual_norm_collection"],
                                   rtol=eps, atol=eps)
        np.testing.assert_allclose(rn, c["expected_residual_norm"], rtol=eps)


@pytest.mark.parametrize("dt", DTYPES)
def test_gmres_solve_krylov(known, dt):
    c = known["gmres_kernels"]["solve_krylov"]
    y = orc.gmres_solve_krylov(to_array(c["residual_norm_collection"], dt),
                               to_array(c["hessenberg"], dt), [2, 2])
    np.testing.assert_allclose(y, c["expected_y"], rtol=np.finfo(dt).eps * 10)


@pytest.mark.parametrize("dt", DTYPES)
def test_solver_known_answers(known, dt):
    dense = {c["name"]: c["dense"] for c in known["solves"]
             if not isinstance(c["dense"], str)}
    r = np.finfo(dt).eps * 10
    for c in known["solves"]:
        d = c["dense"] if not isinstance(c["dense"], str) else dense[c["dense"]]
        rp, ci, v = dense_to_csr(d)
        v = v.astype(dt)
        b = np.array(c["b"], dt)
        if c["solver"] == "cg":
            x, *_ = orc.cg(rp, ci, v, b, jacobi=False,
                           max_iters=c["max_iters"], reduction=r)
        elif c["solver"] == "bicgstab":
            x, *_ = orc.bicgstab(rp, ci, v, b, jacobi=False,
                                 max_iters=c["max_iters"], reduction=r)
        else:
            x, *_ = orc.gmres(rp, ci, v, b, jacobi=False,
                              krylov_dim=c["krylov_dim"],
                              max_iters=c["max_iters"], reduction=r)
        exp = np.array(c["expected"])
        err = np.linalg.norm(x - exp) / max(np.linalg.norm(x), np.linalg.norm(exp))
        tol = (np.sqrt(r) if c.get("tol_sqrt") else r) * c["tol_factor"]
        assert err <= tol, (c["name"], err)


@pytest.mark.parametrize("dt", DTYPES)
def test_batch_bicgstab_logs_iterations(known, dt):
    c = known["batch_bicgstab"]
    n = c["num_rows"]
    d = np.zeros((n, n))
    for i in range(n):
        d[i, i] = c["stencil"][1]
        if i > 0:
            d[i, i - 1] = c["stencil"][0]
        if i < n - 1:
            d[i, i + 1] = c["stencil"][2]
    rp, ci, v = dense_to_csr(d)
    w, s, eci, ev = orc.csr_to_ell(rp, ci, v.astype(dt))
    xs = np.full(n, c["exact_solution"], dt)
    b = (d @ xs).astype(dt)
    x, it, res, conv = orc.batch_bicgstab_ell(n, w, s, eci, ev, b,
                                              max_iters=c["max_iters"],
                                              tol=c["tol"])
    assert conv == 1 and it <= c["max_logged_iters"]
    assert res / np.linalg.norm(b) <= c["tol"]
    assert np.abs(x - xs).max() <= c["tol"] * 10 * 2.5 * 10


def test_cg_poisson_matches_reference_run(known):
    c = known["cg_poisson_2d_256"]
    rp, ci, v = stencils.poisson_2d_5pt(c["grid"])
    xt = std_uniform(c["seed"], len(rp) - 1, -1.0, 1.0)
    b = orc.csr_spmv(rp, ci, v, xt)
    x, it, res, conv = orc.cg(rp, ci, v, b, jacobi=True, max_iters=1000,
                              reduction=1e-10)
    assert it == c["iterations"]
    rel = res[0] / np.linalg.norm(b)
    assert abs(rel - c["relative_residual"]) <= 1e-3 * c["relative_residual"]


def test_ell_sellp_match_csr_random():
    rng = np.random.default_rng(42)
    rp, ci, v = stencils.power_law(3000, seed=3, mu=1.5, max_len=200)
    x = rng.standard_normal((3000, 3))
    y = orc.csr_spmv(rp, ci, v, x)
    w, s, eci, ev = orc.csr_to_ell(rp, ci, v)
    np.testing.assert_allclose(orc.ell_spmv(3000, w, s, eci, ev, x), y, rtol=1e-12, atol=1e-12)
    sets, lens, sci, sv = orc.csr_to_sellp(rp, ci, v, 32, 1)
    np.testing.assert_allclose(orc.sellp_spmv(3000, 32, sets, lens, sci, sv, x), y,
                               rtol=1e-12, atol=1e-12)
    trp, tci, tv = orc.csr_transpose(rp, ci, v, 3000)
    dense = np.zeros((3000, 3000))
    dense[np.repeat(np.arange(3000), np.diff(rp)), ci] = v
    np.testing.assert_allclose(orc.csr_spmv(trp, tci, tv, x), dense.T @ x,
                               rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("ortho", ["cgs", "cgs2"])
def test_gmres_orthogonalisations_meet_known_answers(known, ortho):
    # reference/test/solver/gmres_kernels.cpp:777-812 solves with every
    # ortho_method; the oracle's CGS and CGS2 meet the GMRES known answers
    dense = {c["name"]: c["dense"] for c in known["solves"]
             if not isinstance(c["dense"], str)}
    r = np.finfo(np.float64).eps * 10
    for c in known["solves"]:
        if c["solver"] != "gmres":
            continue
        d = c["dense"] if not isinstance(c["dense"], str) else dense[c["dense"]]
        rp, ci, v = dense_to_csr(d)
        x, *_ = orc.gmres(rp, ci, v, np.array(c["b"]), jacobi=False,
                          krylov_dim=c["krylov_dim"], max_iters=c["max_iters"],
                          reduction=r, ortho=ortho)
        exp = np.array(c["expected"])
        err = np.linalg.norm(x - exp) / max(np.linalg.norm(x), np.linalg.norm(exp))
        tol = (np.sqrt(r) if c.get("tol_sqrt") else r) * c["tol_factor"]
        assert err <= tol, (c["name"], ortho, err)


def test_residual_modes_of_the_oracle():
    # the three baselines and the implicit norm change when CG stops:
    # ||r_k|| <= red * baseline with baseline ||b||, ||r_0|| or 1
    from ginkgo_b200 import stencils
    rp, ci, v = stencils.poisson_2d_5pt(24)
    n = len(rp) - 1
    rng = np.random.default_rng(3)
    b = rng.standard_normal(n)
    x0 = 5 * rng.standard_normal(n)
    r0 = np.linalg.norm(b - orc.csr_spmv(rp, ci, v, x0))
    for mode, base in ((0, np.linalg.norm(b)), (1, r0), (2, 1.0)):
        red = 1e-8 if mode != 2 else 1e-6
        x, it, res, conv = orc.cg(rp, ci, v, b, x0=x0, max_iters=2000, reduction=red,
                                  mode=mode)
        assert conv == 1
        assert res[0] <= red * base
        # one iteration fewer does not meet the goal
        _, it2, res2, conv2 = orc.cg(rp, ci, v, b, x0=x0, max_iters=it - 1,
                                     reduction=red, mode=mode)
        assert conv2 == 0 and res2[0] > red * base
    # ImplicitResidualNorm stops on sqrt(r^T z), not on ||r||
    _, it_i, _, conv_i = orc.cg(rp, ci, v, b, x0=x0, max_iters=2000, reduction=1e-8,
                                mode=orc.IMPLICIT)
    _, it_e, _, _ = orc.cg(rp, ci, v, b, x0=x0, max_iters=2000, reduction=1e-8, mode=0)
    assert conv_i == 1 and it_i != it_e


def test_cg_block_oracle():
    # unit blocks reproduce the scalar-Jacobi CG bit for bit; blocks of 4
    # consecutive rows converge to the explicit residual goal
    from oracle import jacobi as J
    rp, ci, v = stencils.poisson_3d_7pt(8)
    n = len(rp) - 1
    b = np.random.default_rng(1).standard_normal(n)
    _, inv = J.generate(rp, ci, v, 1)
    x1, i1, _, _ = orc.cg(rp, ci, v, b, max_iters=500, reduction=1e-10)
    x2, i2, _, c2 = orc.cg_block(rp, ci, v, b, np.arange(n + 1), [np.array([[d]]) for d in inv],
                                 1, max_iters=500, reduction=1e-10)
    assert i1 == i2 and c2 == 1 and np.array_equal(x1, x2)
    ptrs = list(range(0, n + 1, 4))
    _, bp, blocks = J.generate(rp, ci, v, 4, block_ptrs=ptrs)
    x3, i3, _, c3 = orc.cg_block(rp, ci, v, b, bp, blocks, 4, max_iters=500, reduction=1e-10)
    r = b - orc.csr_spmv(rp, ci, v, x3)
    assert c3 == 1 and i3 <= i1 and np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)


def test_bicgstab_and_gmres_block_oracles():
    # unit blocks reproduce the scalar-Jacobi solvers bit for bit; blocks of
    # four rows converge to the explicit residual goal
    from oracle import jacobi as J
    rp, ci, v = stencils.convection_diffusion_2d(30, 30, 1.0, 0.6, -0.3)
    n = len(rp) - 1
    b = np.random.default_rng(1).standard_normal(n)
    _, inv = J.generate(rp, ci, v, 1)
    unit = [np.array([[d]]) for d in inv]
    x1, i1, _, _ = orc.bicgstab(rp, ci, v, b, max_iters=500, reduction=1e-10)
    x2, i2, _, c2 = orc.bicgstab_block(rp, ci, v, b, np.arange(n + 1), unit, 1,
                                       max_iters=500, reduction=1e-10)
    assert i1 == i2 and c2 == 1 and np.array_equal(x1, x2)
    g1, j1, _, _ = orc.gmres(rp, ci, v, b, krylov_dim=20, max_iters=500, reduction=1e-10)
    g2, j2, _, c3 = orc.gmres_block(rp, ci, v, b, np.arange(n + 1), unit, 1, krylov_dim=20,
                                    max_iters=500, reduction=1e-10)
    assert j1 == j2 and c3 == 1 and np.array_equal(g1, g2)
    ptrs = list(range(0, n + 1, 4))
    _, bp, blocks = J.generate(rp, ci, v, 4, block_ptrs=ptrs)
    for solve in (orc.bicgstab_block, orc.gmres_block):
        x, _, _, conv = solve(rp, ci, v, b, bp, blocks, 4, max_iters=500, reduction=1e-10)
        r = b - orc.csr_spmv(rp, ci, v, x)
        assert conv == 1 and np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)
