"""Differentiable sparse solve x = A^-1 b as a torch.autograd.Function.

Forward: CG with scalar Jacobi (A symmetric positive definite) or BiCGStab
on the device.  Backward, from the converged x only (no stored iterates):
    lambda = A^-T g        (the adjoint solve on a transposed Csr built on
                            the GPU; g = dL/dx)
    dL/db = lambda
    dL/dA = -lambda x^T    on A's pattern (SDDMM kernel)
so gradients flow to whatever produced A's values (for the conductivity
operator, torch autograd carries dL/dA to dL/dtheta through the assembly).
The reference has no autograd path; this is new on the B200 path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import stencils
from ._lib import call
from .matrix import Csr, CudaExecutor, _p, _stream
from .solver import Bicgstab, Cg, Iteration, Jacobi, ResidualNorm


def _solve(A: Csr, b, kind, max_iters, tol):
    fac = Cg if kind == "cg" else Bicgstab
    s = (fac.build()
         .with_criteria(Iteration.build().with_max_iters(max_iters),
                        ResidualNorm.build().with_reduction_factor(tol))
         .with_preconditioner(Jacobi.build().with_max_block_size(1))
         .on(A.exec).generate(A))
    x = torch.zeros_like(b)
    s.apply(b, x)
    if not s.logger.has_converged:
        raise RuntimeError(f"{kind} did not reach {tol} in {max_iters} iterations "
                           f"(residual {s.logger.residual_norm})")
    return x, s.logger


class SparseSolve(torch.autograd.Function):
    """x = A(values)^-1 b on a fixed Csr pattern (row_ptrs, col_idxs)."""

    @staticmethod
    def forward(ctx, values, b, row_ptrs, col_idxs, opts):
        n = row_ptrs.numel() - 1
        exe = CudaExecutor.create(values.device.index or 0)
        A = Csr(exe, (n, n), row_ptrs, col_idxs, values.detach().contiguous())
        b2 = b.detach().contiguous()
        x, log = _solve(A, b2, opts["kind"], opts["max_iters"], opts["tol"])
        ctx.A = A
        ctx.opts = opts
        ctx.forward_iterations = log.num_iterations
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        A = ctx.A
        At = A.transpose()  # GPU count / scan / scatter
        lam, _ = _solve(At, g.contiguous(), ctx.opts["kind"],
                        ctx.opts["max_iters"], ctx.opts["tol"])
        grad_values = None
        if ctx.needs_input_grad[0]:
            grad_values = torch.empty_like(A.values)
            k = 1 if x.dim() == 1 else x.shape[1]
            lam2 = lam.reshape(A.shape[0], k)
            x2 = x.reshape(A.shape[0], k)
            sfx = "f64" if A.dtype == torch.float64 else "f32"
            call(f"b2s_csr_sddmm_{sfx}", A.shape[0], _p(A.row_ptrs),
                 _p(A.col_idxs), A.max_row_nnz, _p(lam2), lam2.stride(0),
                 _p(x2), x2.stride(0), k, -1.0, _p(grad_values),
                 _stream(grad_values))
        grad_b = lam if ctx.needs_input_grad[1] else None
        return grad_values, grad_b, None, None, None


def sparse_solve(values, b, row_ptrs, col_idxs, kind="cg", max_iters=5000,
                 tol=1e-12):
    """Differentiable x = A^-1 b; values follow the Csr pattern."""
    return SparseSolve.apply(values, b, row_ptrs, col_idxs,
                             {"kind": kind, "max_iters": max_iters, "tol": tol})


class ConductivityOperator:
    """The 3D 7-point variable-conductivity operator A(theta) on an nx^3 grid
    with Dirichlet boundary: A_ij = -theta_e for the edge e = (i, j),
    A_ii = sum of theta over the edges at i.  values(theta) assembles the Csr
    values with torch ops, so autograd carries dL/dA to dL/dtheta."""

    def __init__(self, nx: int, device="cuda"):
        self.nx = nx
        n = nx ** 3
        ei, ej = stencils.conductivity_edges(nx)
        self.num_edges = len(ei)
        rp, ci, _ = stencils.conductivity_matrix(nx, np.ones(len(ei)))
        self.n = n
        self.row_ptrs = torch.from_numpy(rp).to(device)
        self.col_idxs = torch.from_numpy(ci).to(device)
        rows = np.repeat(np.arange(n), np.diff(rp))
        key = rows.astype(np.int64) * n + ci
        inner = ej >= 0
        # position of every off-diagonal entry (both orientations)
        pos_ij = np.searchsorted(key, ei[inner] * n + ej[inner])
        pos_ji = np.searchsorted(key, ej[inner] * n + ei[inner])
        diag_pos = np.searchsorted(key, np.arange(n, dtype=np.int64) * (n + 1))
        inner_ids = np.nonzero(inner)[0]
        off_pos = np.concatenate([pos_ij, pos_ji])
        off_edge = np.concatenate([inner_ids, inner_ids])
        # diagonal gets theta of every edge at the node
        d_pos = np.concatenate([diag_pos[ei], diag_pos[ej[inner]]])
        d_edge = np.concatenate([np.arange(len(ei)), inner_ids])
        self._off_pos = torch.from_numpy(off_pos).to(device)
        self._off_edge = torch.from_numpy(off_edge).to(device)
        self._d_pos = torch.from_numpy(d_pos).to(device)
        self._d_edge = torch.from_numpy(d_edge).to(device)
        self.nnz = len(ci)

    def values(self, theta: torch.Tensor) -> torch.Tensor:
        v = torch.zeros(self.nnz, dtype=theta.dtype, device=theta.device)
        v = v.index_add(0, self._off_pos, -theta[self._off_edge])
        v = v.index_add(0, self._d_pos, theta[self._d_edge])
        return v

    def solve(self, theta, b, **kw):
        return sparse_solve(self.values(theta), b, self.row_ptrs, self.col_idxs, **kw)
