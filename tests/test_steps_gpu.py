"""Kernel-level Krylov steps (the drop-ins for a caller that keeps the
reference's own loop) against the reference's known answers and the
oracle's restatement of the same kernels."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import to_array
from ginkgo_b200._lib import call
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DT = [(torch.float64, "f64"), (torch.float32, "f32")]


_KEEP = []


def P(t):
    # keep the tensor alive until the test ends: a temporary freed before
    # the call would hand its memory to the next allocation
    _KEEP.append(t)
    return C.c_void_p(t.data_ptr())


def S():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a, dt):
    return torch.tensor(np.asarray(a, dtype=np.float64), dtype=dt, device="cuda")


STOPPED = 0x01 | 0x40  # stopped by criterion 1, finalized


@pytest.mark.parametrize("dt,s", DT)
def test_cg_steps_known_answers(known, dt, s):
    kc = known["cg_kernels"]
    for key in ("step_1", "step_1_div_by_zero"):
        c = kc[key]
        p = torch.full((2, 2), c["p"], dtype=dt, device="cuda")
        z = torch.full((2, 2), c["z"], dtype=dt, device="cuda")
        st = torch.tensor([STOPPED if f else 0 for f in c["stopped"]],
                          dtype=torch.uint8, device="cuda")
        call(f"b2s_cg_step_1_{s}", 2, 2, P(p), 2, P(z), 2, P(dev(c["rho"], dt)),
             P(dev(c["prev_rho"], dt)), P(st), S())
        assert np.array_equal(p.cpu().numpy(), np.array(c["expected_p"]))
    for key in ("step_2", "step_2_div_by_zero"):
        c = kc[key]
        x = torch.full((2, 2), c["x"], dtype=dt, device="cuda")
        r = torch.full((2, 2), c["r"], dtype=dt, device="cuda")
        p = torch.full((2, 2), c["p"], dtype=dt, device="cuda")
        q = torch.full((2, 2), c["q"], dtype=dt, device="cuda")
        st = torch.tensor([STOPPED if f else 0 for f in c["stopped"]],
                          dtype=torch.uint8, device="cuda")
        call(f"b2s_cg_step_2_{s}", 2, 2, P(x), 2, P(r), 2, P(p), 2, P(q), 2,
             P(dev(c["beta"], dt)), P(dev(c["rho"], dt)), P(st), S())
        assert np.array_equal(x.cpu().numpy(), np.array(c["expected_x"]))
        assert np.array_equal(r.cpu().numpy(), np.array(c["expected_r"]))


@pytest.mark.parametrize("dt,s", DT)
def test_cg_initialize(dt, s):
    b = dev([[2.0, 2.0], [2.0, 2.0]], dt)
    r, z, p, q = (torch.ones((2, 2), dtype=dt, device="cuda") for _ in range(4))
    prev_rho = torch.zeros(2, dtype=dt, device="cuda")
    rho = torch.ones(2, dtype=dt, device="cuda")
    st = torch.full((2,), STOPPED, dtype=torch.uint8, device="cuda")
    call(f"b2s_cg_initialize_{s}", 2, 2, P(b), 2, P(r), 2, P(z), 2, P(p), 2,
         P(q), 2, P(prev_rho), P(rho), P(st), S())
    assert torch.equal(r, b) and not z.any() and not p.any() and not q.any()
    assert rho.tolist() == [0, 0] and prev_rho.tolist() == [1, 1]
    assert st.tolist() == [0, 0]


@pytest.mark.parametrize("dt,s", DT)
def test_gmres_hessenberg_qr_and_solve_krylov(known, dt, s):
    eps = float(torch.finfo(dt).eps) * 10
    for key in ("hessenberg_qr_iter0", "hessenberg_qr_iter1"):
        c = known["gmres_kernels"][key]
        gs = dev(to_array(c["givens_sin"]), dt)
        gc = dev(to_array(c["givens_cos"]), dt)
        rnc = dev(to_array(c["residual_norm_collection"]), dt)
        h = dev(to_array(c["hessenberg_iter"]), dt)
        rn = torch.full((2,), float("nan"), dtype=dt, device="cuda")
        fin = torch.full((2,), c["iteration"], dtype=torch.int64, device="cuda")
        st = torch.zeros(2, dtype=torch.uint8, device="cuda")
        call(f"b2s_gmres_hessenberg_qr_{s}", 2, c["iteration"], P(gs), 2, P(gc), 2,
             P(rn), P(rnc), 2, P(h), 2, P(fin), P(st), S())
        assert fin.tolist() == [c["iteration"] + 1] * 2
        for got, k in ((gc, "expected_givens_cos"), (gs, "expected_givens_sin"),
                       (h, "expected_hessenberg_iter"),
                       (rnc, "expected_residual_norm_collection")):
            np.testing.assert_allclose(got.cpu().numpy(), np.array(c[k]),
                                       rtol=eps, atol=eps, err_msg=k)
        np.testing.assert_allclose(rn.cpu().numpy(), c["expected_residual_norm"],
                                   rtol=eps)
    c = known["gmres_kernels"]["solve_krylov"]
    h = dev(to_array(c["hessenberg"]), dt)
    rnc = dev(to_array(c["residual_norm_collection"]), dt)
    y = torch.full((2, 2), float("nan"), dtype=dt, device="cuda")
    fin = torch.tensor([2, 2], dtype=torch.int64, device="cuda")
    st = torch.zeros(2, dtype=torch.uint8, device="cuda")
    call(f"b2s_gmres_solve_krylov_{s}", 2, P(rnc), 2, P(h), 6, P(y), 2, P(fin),
         P(st), S())
    np.testing.assert_allclose(y.cpu().numpy(), c["expected_y"], rtol=eps)


@pytest.mark.parametrize("dt,s", DT)
def test_bicgstab_steps_match_formulas(dt, s):
    rng = np.random.default_rng(0)
    n, k = 1000, 3
    npdt = np.float64 if dt == torch.float64 else np.float32
    r, p, v, sv, t, y, z, x = (rng.standard_normal((n, k)).astype(npdt) for _ in range(8))
    rho, prev, alpha, omega, beta, gamma = (rng.uniform(0.5, 2, k).astype(npdt)
                                            for _ in range(6))
    prev[1] = 0  # p = r branch
    stat = np.array([0, 0, STOPPED], np.uint8)
    D = {nm: torch.from_numpy(a.copy()).cuda() for nm, a in
         dict(r=r, p=p, v=v, s=sv, t=t, y=y, z=z, x=x, rho=rho, prev=prev,
              alpha=alpha, omega=omega, beta=beta, gamma=gamma).items()}
    st = torch.from_numpy(stat).cuda()
    call(f"b2s_bicgstab_step_1_{s}", n, k, P(D["r"]), k, P(D["p"]), k, P(D["v"]), k,
         P(D["rho"]), P(D["prev"]), P(D["alpha"]), P(D["omega"]), P(st), S())
    exp_p = p.copy()
    for j in range(2):
        if prev[j] * omega[j] != 0:
            exp_p[:, j] = r[:, j] + rho[j] / prev[j] * alpha[j] / omega[j] * (
                p[:, j] - omega[j] * v[:, j])
        else:
            exp_p[:, j] = r[:, j]
    # FMA contraction on the GPU: a few ulps of the largest term
    np.testing.assert_allclose(D["p"].cpu().numpy(), exp_p, rtol=1e-5 if s == "f32" else 1e-13,
                               atol=1e-5 if s == "f32" else 1e-14)
    call(f"b2s_bicgstab_step_2_{s}", n, k, P(D["r"]), k, P(D["s"]), k, P(D["v"]), k,
         P(D["rho"]), P(D["alpha"]), P(D["beta"]), P(st), S())
    a2 = rho / beta
    exp_s = sv.copy()
    exp_s[:, :2] = r[:, :2] - a2[:2] * v[:, :2]
    np.testing.assert_allclose(D["s"].cpu().numpy(), exp_s, rtol=1e-5 if s == "f32" else 1e-13,
                               atol=1e-5 if s == "f32" else 1e-13)
    np.testing.assert_allclose(D["alpha"].cpu().numpy()[:2], a2[:2], rtol=1e-6)
    # finalize: only stopped-and-not-finalized columns change
    st2 = torch.tensor([0x01, 0, STOPPED], dtype=torch.uint8, device="cuda")
    x0 = D["x"].clone()
    call(f"b2s_bicgstab_finalize_{s}", n, k, P(D["x"]), k, P(D["y"]), k,
         P(D["alpha"]), P(st2), S())
    xf = D["x"].cpu().numpy()
    ag = D["alpha"].cpu().numpy()
    # the GPU contracts x + alpha y into one fused multiply-add
    np.testing.assert_allclose(xf[:, 0], x0.cpu().numpy()[:, 0] + ag[0] * y[:, 0],
                               rtol=1e-5 if s == "f32" else 1e-13,
                               atol=1e-5 if s == "f32" else 1e-15)
    assert np.array_equal(xf[:, 1:], x0.cpu().numpy()[:, 1:])
    assert st2.tolist() == [0x41, 0, STOPPED]


@pytest.mark.parametrize("dt,s", DT)
def test_dense_dot_norm_and_residual_check(dt, s):
    from ginkgo_b200._lib import lib
    rng = np.random.default_rng(1)
    n, k = 100001, 4
    a = torch.from_numpy(rng.standard_normal((n, k))).to(dt).cuda()
    b = torch.from_numpy(rng.standard_normal((n, k))).to(dt).cuda()
    wsb = lib().b2s_dense_reduction_workspace_bytes(k, a.element_size())
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dot = torch.empty(k, dtype=dt, device="cuda")
    nrm = torch.empty(k, dtype=dt, device="cuda")
    call(f"b2s_dense_compute_dot_{s}", n, k, P(a), k, P(b), k, P(dot), P(ws), wsb, S())
    call(f"b2s_dense_compute_norm2_{s}", n, k, P(a), k, P(nrm), P(ws), wsb, S())
    A, B = a.double().cpu().numpy(), b.double().cpu().numpy()
    tol = 1e-12 if s == "f64" else 2e-4
    np.testing.assert_allclose(dot.cpu().numpy(), (A * B).sum(0), rtol=tol, atol=tol * 300)
    np.testing.assert_allclose(nrm.cpu().numpy(), np.linalg.norm(A, axis=0), rtol=tol)
    # residual_norm: columns 0, 2 converge; column 3 was stopped already
    tau = dev([1e-11, 1.0, 2e-11, 5.0], dt)
    orig = dev([1.0, 1.0, 1.0, 1.0], dt)
    st = torch.tensor([0, 0, 0, STOPPED], dtype=torch.uint8, device="cuda")
    flags = torch.zeros(2, dtype=torch.int32, device="cuda")
    call(f"b2s_residual_norm_check_{s}", 4, P(tau), P(orig), 1e-10, 1, 1, P(st),
         P(flags), S())
    assert st.tolist() == [0xC1, 0, 0xC1, STOPPED]
    assert flags.tolist() == [0, 1]  # column 1 still running; one changed
