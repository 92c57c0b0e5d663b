"""Pure-Python restatement of the reference's CB-GMRES (compressed-basis
GMRES, core/solver/cb_gmres.cpp with reference/solver/cb_gmres_kernels.cpp
and core/solver/cb_gmres_accessor.hpp) — TEST INFRASTRUCTURE ONLY.

The checker for a future device CB-GMRES: restarted GMRES whose Krylov basis
is stored in a reduced format and read back for the orthogonalisation and
the solution update, while the next vector, the Hessenberg matrix and the
Givens rotations stay in the value type.  Pinned by the reference's own
solve tests (reference/test/solver/cb_gmres_kernels.cpp).  Only tests import
this module.

Storage formats (cb_gmres.cpp:100-157, the storage_precision enum):
  keep      the value type
  reduce1   one precision down (double -> float, float -> half)
  reduce2   two down (double -> half, float -> half)
  integer   a scaled integer of the value type's width (double -> int64,
            float -> int32)
  ireduce1  a scaled integer one width down (double -> int32, float -> int16)
  ireduce2  two widths down (double -> int16, float -> int16)
A scaled integer stores v / s truncated toward zero and reads int * s, with
one scale s per basis vector and right-hand side, set to
(max|v| / ||v||) * 2 / INT_MAX when the vector is written (accessor.hpp:
137-152, finish_arnoldi_CGS, restart).
"""
from __future__ import annotations

import numpy as np

_FLOAT = {"f64": np.float64, "f32": np.float32}
_STORE = {
    "f64": {"keep": np.float64, "reduce1": np.float32, "reduce2": np.float16,
            "integer": np.int64, "ireduce1": np.int32, "ireduce2": np.int16},
    "f32": {"keep": np.float32, "reduce1": np.float16, "reduce2": np.float16,
            "integer": np.int32, "ireduce1": np.int16, "ireduce2": np.int16},
}


class _Basis:
    """The (krylov_dim + 1) x n x k basis through the reference's accessor:
    reduced_row_major for floating storage, scaled_reduced_row_major (scale
    per vector and column) for integer storage."""

    def __init__(self, vt, st, dim, n, k):
        self.vt, self.st = vt, st
        self.scaled = np.issubdtype(st, np.integer)
        self.data = np.zeros((dim, n, k), dtype=st)
        self.scale = np.ones((dim, k), dtype=vt)
        self.corr = (vt(2) / vt(np.iinfo(st).max)) if self.scaled else vt(1)

    def write_scalar(self, v, i, value):
        if self.scaled:
            self.scale[v, i] = self.vt(value) * self.corr

    def write(self, v, i, col):  # col: value-type vector
        if self.scaled:
            q = (col / self.scale[v, i]).astype(self.vt)
            self.data[v, :, i] = np.trunc(q).astype(self.st)
        else:
            self.data[v, :, i] = col.astype(self.st)

    def read(self, v, i):
        x = self.data[v, :, i].astype(self.vt)
        return x * self.scale[v, i] if self.scaled else x


def _dot(a, b, vt):
    s = vt(0)
    for x, y in zip(a, b):  # sequential, as the reference loop
        s = vt(s + vt(x) * vt(y))
    return s


def _norm2(a, vt):
    s = vt(0)
    for x in a:
        s = vt(s + vt(x) * vt(x))
    return vt(np.sqrt(s))


def _finish_arnoldi_cgs(nk, basis, hess, arn, it, stopped, vt):
    """finish_arnoldi_CGS (reference/solver/cb_gmres_kernels.cpp:30-139):
    CGS, re-orthogonalised (at most twice more) while the norm drops below
    eta = 1/sqrt(2) of the previous one."""
    eta = vt(1.0 / np.sqrt(2.0))
    n, k = nk.shape
    for i in range(k):
        arn[0, i] = eta * _norm2(nk[:, i], vt)
        if stopped[i]:
            continue
        for m in range(it + 1):
            hess[m, i] = _dot(nk[:, i], basis.read(m, i), vt)
        for m in range(it + 1):
            nk[:, i] = (nk[:, i] - hess[m, i] * basis.read(m, i)).astype(vt)
        arn[1, i] = _norm2(nk[:, i], vt)
        arn[2, i] = np.max(np.abs(nk[:, i])) if basis.scaled else vt(0)
        l = 1
        while arn[1, i] < arn[0, i] and l < 3:
            arn[0, i] = eta * arn[1, i]
            buf = [_dot(nk[:, i], basis.read(m, i), vt) for m in range(it + 1)]
            for m in range(it + 1):
                nk[:, i] = (nk[:, i] - buf[m] * basis.read(m, i)).astype(vt)
                hess[m, i] = vt(hess[m, i] + buf[m])
            arn[1, i] = _norm2(nk[:, i], vt)
            arn[2, i] = np.max(np.abs(nk[:, i]))
            l += 1
        basis.write_scalar(it + 1, i, vt(arn[2, i] / arn[1, i]))
        hess[it + 1, i] = arn[1, i]
        nk[:, i] = (nk[:, i] / hess[it + 1, i]).astype(vt)
        basis.write(it + 1, i, nk[:, i])


def _givens(gs, gc, hess, it, stopped, vt):
    """givens_rotation + calculate_sin_and_cos (:142-197)."""
    for i in range(hess.shape[1]):
        if stopped[i]:
            continue
        for j in range(it):
            t = vt(gc[j, i] * hess[j, i] + gs[j, i] * hess[j + 1, i])
            hess[j + 1, i] = vt(-gs[j, i] * hess[j, i] + gc[j, i] * hess[j + 1, i])
            hess[j, i] = t
        if hess[it, i] == 0:
            gc[it, i], gs[it, i] = vt(0), vt(1)
        else:
            a, b = hess[it, i], hess[it + 1, i]
            scale = vt(abs(a) + abs(b))
            hyp = vt(scale * np.sqrt(vt(abs(a / scale) * abs(a / scale) +
                                        abs(b / scale) * abs(b / scale))))
            gc[it, i], gs[it, i] = vt(a / hyp), vt(b / hyp)
        hess[it, i] = vt(gc[it, i] * hess[it, i] + gs[it, i] * hess[it + 1, i])
        hess[it + 1, i] = vt(0)


def _apply_prec(prec, v):
    return v if prec is None else prec(v)


def solve(A, b, x0=None, value_type="f64", storage="keep", krylov_dim=100,
          max_iters=100, reduction_factor=None, preconditioner=None):
    """CbGmres<ValueType>::apply_dense_impl (core/solver/cb_gmres.cpp:
    208-484) with stop::Iteration(max_iters) and stop::ResidualNorm
    (baseline initial_resnorm, reduction_factor; default 10 eps of the
    value type, as the tests use).  A: dense n x n; b: n or n x k.
    preconditioner: None (identity) or a function v -> M v on n x k arrays.
    Returns (x, total_iterations)."""
    vt = _FLOAT[value_type]
    st = _STORE[value_type][storage]
    A = np.asarray(A, dtype=vt)
    b = np.asarray(b, dtype=vt)
    one_col = b.ndim == 1
    b = b.reshape(len(b), -1)
    n, k = b.shape
    x = np.zeros_like(b) if x0 is None else np.asarray(x0, dtype=vt).reshape(n, k).copy()
    red = vt(10 * np.finfo(vt).eps) if reduction_factor is None else vt(reduction_factor)
    basis = _Basis(vt, st, krylov_dim + 1, n, k)
    hessenberg = np.zeros((krylov_dim + 1, krylov_dim, k), dtype=vt)
    gs = np.zeros((krylov_dim, k), dtype=vt)
    gc = np.zeros((krylov_dim, k), dtype=vt)
    rnc = np.zeros((krylov_dim + 1, k), dtype=vt)
    rnorm = np.zeros(k, dtype=vt)
    arn = np.zeros((3, k), dtype=vt)
    final_iter = np.zeros(k, dtype=np.int64)

    def matvec(v):
        out = np.zeros_like(v)
        for c in range(v.shape[1]):
            for r in range(n):
                out[r, c] = _dot(A[r], v[:, c], vt)
        return out

    def restart(res):
        """restart (:292-354)."""
        nk = np.zeros_like(res)
        for j in range(k):
            rnorm[j] = _norm2(res[:, j], vt)
            arn[2, j] = np.max(np.abs(res[:, j])) if basis.scaled else vt(0)
            basis.write_scalar(0, j, vt(arn[2, j] / rnorm[j]))
            rnc[:, j] = 0
            rnc[0, j] = rnorm[j]
            v0 = (res[:, j] / rnorm[j]).astype(vt)
            basis.write(0, j, v0)
            nk[:, j] = v0
            final_iter[j] = 0
        for m in range(1, krylov_dim + 1):
            for j in range(k):
                basis.write_scalar(m, j, vt(1))
                basis.write(m, j, np.zeros(n, dtype=vt))
        return nk

    def solve_krylov(iters):
        """solve_upper_triangular + calculate_qy (:222-266)."""
        before = np.zeros((n, k), dtype=vt)
        for c in range(k):
            m = int(final_iter[c])
            y = np.zeros(m, dtype=vt)
            for i in range(m - 1, -1, -1):
                t = rnc[i, c]
                for j in range(i + 1, m):
                    t = vt(t - hessenberg[i, j, c] * y[j])
                y[i] = vt(t / hessenberg[i, i, c])
            for j in range(m):
                before[:, c] = (before[:, c] + basis.read(j, c) * y[j]).astype(vt)
        return before

    residual = (b - matvec(x)).astype(vt)
    nk = restart(residual)
    baseline = np.array([_norm2(residual[:, j], vt) for j in range(k)], dtype=vt)
    stopped = np.zeros(k, bool)
    converged = np.zeros(k, bool)
    total_iter, restart_iter = -1, 0
    stop_encountered = np.zeros(k, bool)
    fully_converged = np.zeros(k, bool)
    start_force_reset = 10
    perform_reset = False
    forced_fraction = 10
    forced_limit = krylov_dim // forced_fraction
    forced_iterations = forced_limit
    while True:
        total_iter += 1
        if forced_iterations < forced_limit and \
                forced_iterations < total_iter // forced_fraction:
            forced_iterations += 1
        else:
            # stop::Iteration, then stop::ResidualNorm on the implicit norm
            one_changed = False
            for j in range(k):
                if stopped[j]:
                    continue
                if total_iter >= max_iters:
                    stopped[j], one_changed = True, True
                elif rnorm[j] <= red * baseline[j]:
                    stopped[j] = converged[j] = one_changed = True
            if one_changed or stopped.all():
                changed = False
                for j in range(k):
                    if fully_converged[j] or not converged[j]:
                        continue
                    if stop_encountered[j] or total_iter < start_force_reset:
                        fully_converged[j] = True
                    else:
                        stop_encountered[j] = True
                        stopped[j] = converged[j] = False
                        changed = True
                if not changed:
                    break
                perform_reset = True
                forced_iterations = 0
            else:
                stop_encountered[:] = False
        if perform_reset or restart_iter == krylov_dim:
            perform_reset = False
            before = solve_krylov(restart_iter)
            x = (x + _apply_prec(preconditioner, before)).astype(vt)
            residual = (b - matvec(x)).astype(vt)
            nk = restart(residual)
            restart_iter = 0
        pv = _apply_prec(preconditioner, nk).astype(vt)
        nk = matvec(pv)
        # arnoldi (:357-391)
        final_iter += (~stopped).astype(np.int64)
        hess_it = hessenberg[:restart_iter + 2, restart_iter, :]
        _finish_arnoldi_cgs(nk, basis, hess_it, arn, restart_iter, stopped, vt)
        _givens(gs, gc, hess_it, restart_iter, stopped, vt)
        for j in range(k):
            if stopped[j]:
                continue
            rnc[restart_iter + 1, j] = vt(-gs[restart_iter, j] * rnc[restart_iter, j])
            rnc[restart_iter, j] = vt(gc[restart_iter, j] * rnc[restart_iter, j])
            rnorm[j] = abs(rnc[restart_iter + 1, j])
        hessenberg[:restart_iter + 2, restart_iter, :] = hess_it
        restart_iter += 1
    before = solve_krylov(restart_iter)
    x = (x + _apply_prec(preconditioner, before)).astype(vt)
    return (x[:, 0] if one_col else x), total_iter

