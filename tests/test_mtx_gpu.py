"""A MatrixMarket file read into Csr, Ell and Sellp on the device and
applied, against a dense product on the host (the reader's parity is
covered on CPU; this checks the file-to-device path)."""
import numpy as np
import pytest
import torch

from ginkgo_b200 import mtx_io as M
from ginkgo_b200 import stencils
from ginkgo_b200.matrix import Csr, CudaExecutor, Ell, Sellp

pytestmark = pytest.mark.gpu


def _symmetric_lower_text(rp, ci, v, n):
    lines = []
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            if ci[k] <= r:
                lines.append(f"{r + 1} {int(ci[k]) + 1} {float(v[k])!r}")
    return ("%%MatrixMarket matrix coordinate real symmetric\n% 7-point 6^3\n"
            f"{n} {n} {len(lines)}\n" + "\n".join(lines) + "\n")


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("kind", [Csr, Ell, Sellp])
def test_mtx_file_to_device_spmv(dtype, kind):
    rp, ci, v = stencils.poisson_3d_7pt(6)
    n = len(rp) - 1
    text = _symmetric_lower_text(rp, ci, v, n)
    dense = np.zeros((n, n))
    for r in range(n):
        dense[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
    exe = CudaExecutor.create(0)
    kw = {"slice_size": 32} if kind is Sellp else {}
    A = M.read(kind, text, exe, dtype=dtype, **kw)
    x = np.random.default_rng(0).standard_normal(n)
    xd = torch.from_numpy(x).to(dtype).cuda()
    y = torch.empty(n, dtype=dtype, device="cuda")
    A.apply(xd, y)
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    np.testing.assert_allclose(y.cpu().double().numpy(), dense @ x.astype(
        np.float32 if dtype == torch.float32 else np.float64), rtol=tol, atol=tol * 10)


def test_csr_written_back_matches_the_file_entries():
    rp, ci, v = stencils.poisson_3d_7pt(5)
    n = len(rp) - 1
    A = Csr.read(CudaExecutor.create(0), rp, ci, v)
    text = M.write(A)
    d = M.read_raw(text)
    assert d.size == (n, n)
    assert np.array_equal(d.row_idxs, np.repeat(np.arange(n), np.diff(rp)))
    assert np.array_equal(d.col_idxs, ci) and np.array_equal(d.values, v)
