"""The differentiable solve: gradients against a dense FP64 torch solve on an
8^3 instance and against central finite differences on 64 conductivities of
the 64^3 operator; the GPU transpose used by the adjoint against the oracle."""
import numpy as np
import pytest
import torch

from ginkgo_b200.autograd import ConductivityOperator, sparse_solve

pytestmark = pytest.mark.gpu


def _loss(x, xt):
    return ((x - xt) ** 2).sum()


def test_gradient_matches_dense_torch_8cubed():
    torch.manual_seed(0)
    op = ConductivityOperator(8)
    theta = torch.exp(0.5 * torch.randn(op.num_edges, dtype=torch.float64,
                                         device="cuda")).requires_grad_(True)
    b = torch.randn(op.n, 16, dtype=torch.float64, device="cuda", requires_grad=True)
    xt = torch.randn(op.n, 16, dtype=torch.float64, device="cuda")
    x = op.solve(theta, b, tol=1e-14)
    loss = _loss(x, xt)
    loss.backward()
    g_theta, g_b = theta.grad.clone(), b.grad.clone()
    # dense reference: same assembly, torch.linalg.solve, torch autograd
    th2 = theta.detach().clone().requires_grad_(True)
    b2 = b.detach().clone().requires_grad_(True)
    vals = op.values(th2)
    dense = torch.zeros(op.n, op.n, dtype=torch.float64, device="cuda")
    rows = torch.repeat_interleave(torch.arange(op.n, device="cuda"),
                                   torch.diff(op.row_ptrs.long()))
    dense = dense.index_put((rows, op.col_idxs.long()), vals)
    xd = torch.linalg.solve(dense, b2)
    _loss(xd, xt).backward()
    assert torch.allclose(x, xd, rtol=1e-10, atol=1e-12)
    rel_t = (g_theta - th2.grad).norm() / th2.grad.norm()
    rel_b = (g_b - b2.grad).norm() / b2.grad.norm()
    assert rel_t < 1e-9, rel_t
    assert rel_b < 1e-9, rel_b


def test_gradient_matches_central_differences_64cubed():
    """The differentiable-solve workload: 64^3, 16 right-hand sides,
    theta ~ lognormal(0, 0.5); 64 random conductivities checked."""
    g = torch.Generator(device="cuda").manual_seed(1)
    op = ConductivityOperator(64)
    theta = torch.exp(0.5 * torch.randn(op.num_edges, dtype=torch.float64,
                                         device="cuda", generator=g))
    b = torch.randn(op.n, 16, dtype=torch.float64, device="cuda", generator=g)
    xt = torch.randn(op.n, 16, dtype=torch.float64, device="cuda", generator=g)
    th = theta.clone().requires_grad_(True)
    loss = _loss(op.solve(th, b, tol=1e-13), xt)
    loss.backward()
    grad = th.grad
    idx = torch.randperm(op.num_edges, generator=torch.Generator().manual_seed(2))[:64]
    errs = []
    with torch.no_grad():
        for e in idx.tolist():
            h = 1e-4 * float(theta[e])
            tp = theta.clone()
            tp[e] += h
            tm = theta.clone()
            tm[e] -= h
            fd = (_loss(op.solve(tp, b, tol=1e-13), xt) -
                  _loss(op.solve(tm, b, tol=1e-13), xt)) / (2 * h)
            errs.append(abs(float(fd) - float(grad[e])) /
                        max(abs(float(fd)), 1e-3 * float(grad.abs().max())))
    # FD noise: solver tolerance 1e-13 on a loss of ~1e7, divided by 2h
    assert max(errs) < 5e-4, max(errs)


def test_gpu_transpose_used_by_adjoint_matches_oracle():
    from ginkgo_b200 import stencils
    from ginkgo_b200.matrix import Csr, CudaExecutor
    from oracle import oracle as orc
    exe = CudaExecutor.create(0)
    # non-symmetric values on the conductivity pattern
    op = ConductivityOperator(10)
    rp = op.row_ptrs.cpu().numpy()
    ci = op.col_idxs.cpu().numpy()
    v = np.random.default_rng(4).standard_normal(len(ci))
    A = Csr.read(exe, rp, ci, v)
    T = A.transpose()
    trp, tci, tv = orc.csr_transpose(rp, ci, v, len(rp) - 1)
    np.testing.assert_array_equal(T.row_ptrs.cpu().numpy(), trp)
    np.testing.assert_array_equal(T.col_idxs.cpu().numpy(), tci)
    np.testing.assert_array_equal(T.values.cpu().numpy(), tv)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("k", [1, 3, 4, 8, 16])
def test_sddmm_matches_dense_sampling(dt, k):
    """out[e] = alpha u(row_e, :) . w(col_e, :) on a Csr pattern: the
    subwarp kernel (narrow blocks) and the 16-byte lane kernel (k * value
    size a multiple of 32 bytes) against numpy in FP64."""
    from ginkgo_b200 import stencils
    from ginkgo_b200._lib import call
    from ginkgo_b200.matrix import _p, _stream
    rp, ci, _ = stencils.power_law(3000, seed=4, mu=2.0, max_len=200)
    n = len(rp) - 1
    rng = np.random.default_rng(k)
    u = rng.standard_normal((n, k))
    w = rng.standard_normal((n, k))
    npdt = np.float64 if dt == torch.float64 else np.float32
    ud = torch.from_numpy(u.astype(npdt)).cuda()
    wd = torch.from_numpy(w.astype(npdt)).cuda()
    out = torch.empty(len(ci), dtype=dt, device="cuda")
    rpd = torch.from_numpy(rp).cuda()
    cid = torch.from_numpy(ci).cuda()
    sfx = "f64" if dt == torch.float64 else "f32"
    call(f"b2s_csr_sddmm_{sfx}", n, _p(rpd), _p(cid), int(np.diff(rp).max()), _p(ud), k,
         _p(wd), k, k, -0.5, _p(out), _stream(out))
    rows = np.repeat(np.arange(n), np.diff(rp))
    uq, wq = u.astype(npdt).astype(np.float64), w.astype(npdt).astype(np.float64)
    ref = -0.5 * np.einsum("ij,ij->i", uq[rows], wq[ci])
    scale = 0.5 * np.einsum("ij,ij->i", np.abs(uq[rows]), np.abs(wq[ci]))
    tol = 1e-14 if dt == torch.float64 else 1e-6
    assert (np.abs(out.cpu().numpy() - ref) / scale).max() <= tol
