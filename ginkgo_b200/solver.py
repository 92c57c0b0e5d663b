"""Solver factories over the fused C-ABI solvers, named after the
reference's ``gko::solver`` / ``gko::stop`` / ``gko::preconditioner`` API:

    solver = (Cg.build()
              .with_criteria(Iteration.build().with_max_iters(1000),
                             ResidualNorm.build().with_reduction_factor(1e-10))
              .with_preconditioner(Jacobi.build().with_max_block_size(1))
              .on(exec)
              .generate(A))
    solver.apply(b, x)                # x holds the initial guess
    solver.logger.num_iterations      # like gko::log::Convergence

Scalar Jacobi (max_block_size 1) and block Jacobi (2..32) are fused into
every solver; stopping is Iteration plus one residual criterion, ResidualNorm
(baselines rhs_norm, initial_resnorm, absolute) or, for CG and BiCGStab,
ImplicitResidualNorm (include/ginkgo/core/stop/residual_norm.hpp).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import GinkgoError, call, lib
from .matrix import Csr, _check_dense, _p, _stream

_SFX = {torch.float64: "f64", torch.float32: "f32"}
# gmres::ortho_method (include/ginkgo/core/solver/gmres.hpp:38-50) as the C
# ABI's B2S_ORTHO_* values
_ORTHO = {"mgs": 0, "cgs": 1, "cgs2": 2}
# cb_gmres::storage_precision (include/ginkgo/core/solver/cb_gmres.hpp:38-67)
# of CbGmres<double> as the C ABI's GMRES variants (keep is plain FP64 GMRES)
_CB_STORAGE = {"keep": 0, "reduce1": 3, "reduce2": 4, "integer": 5, "ireduce1": 6,
               "ireduce2": 7}


# --------------------------------------------------------------- criteria --
class _Builder:
    """Generic ``X.build().with_a(v).with_b(w)`` parameter builder."""

    def __init__(self, cls, **defaults):
        self._cls = cls
        self._params = dict(defaults)

    def __getattr__(self, name):
        if name.startswith("with_"):
            key = name[5:]

            def setter(*args):
                self._params[key] = args[0] if len(args) == 1 else args
                return self
            return setter
        raise AttributeError(name)

    def on(self, exec_):
        return self._cls(exec_, **self._params)

    def params(self):
        return dict(self._params)


class Iteration:
    """stop::Iteration (core/stop/iteration.cpp:14-24)."""

    @staticmethod
    def build():
        return _Builder(Iteration, max_iters=0)

    def __init__(self, exec_=None, max_iters=0):
        self.max_iters = int(max_iters)


# stop::mode (include/ginkgo/core/stop/residual_norm.hpp:37) as the C ABI's
# B2S_BASELINE_* values; B2S_STOP_IMPLICIT marks ImplicitResidualNorm
_BASELINES = {"rhs_norm": 0, "initial_resnorm": 1, "absolute": 2}
_STOP_IMPLICIT = 4


class ResidualNorm:
    """stop::ResidualNorm (core/stop/residual_norm.cpp:95-230):
    ||r|| <= reduction_factor * baseline, baseline ||b|| (rhs_norm, the
    default), ||b - A x_0|| (initial_resnorm) or 1 (absolute)."""
    implicit = False

    @staticmethod
    def build():
        return _Builder(ResidualNorm, reduction_factor=1e-15, baseline="rhs_norm")

    def __init__(self, exec_=None, reduction_factor=1e-15, baseline="rhs_norm"):
        if baseline not in _BASELINES:
            raise ValueError(f"unknown baseline {baseline!r}: one of {sorted(_BASELINES)}")
        self.reduction_factor = float(reduction_factor)
        self.baseline = baseline

    @property
    def mode(self):
        return _BASELINES[self.baseline] | (_STOP_IMPLICIT if self.implicit else 0)


class ImplicitResidualNorm(ResidualNorm):
    """stop::ImplicitResidualNorm (include/ginkgo/core/stop/residual_norm.hpp:175,
    core/stop/residual_norm.cpp:205-225): sqrt|rho| <= reduction_factor *
    baseline, rho the solver's implicit squared residual norm (r^T z in CG,
    r_hat^T r in BiCGStab)."""
    implicit = True

    @staticmethod
    def build():
        return _Builder(ImplicitResidualNorm, reduction_factor=1e-15, baseline="rhs_norm")


def _criteria(crits):
    """(max_iters, reduction_factor, residual_mode) of a criterion list: an
    Iteration criterion and at most one residual criterion."""
    max_iters, res = None, None
    for c in crits:
        if isinstance(c, _Builder):
            c = c.on(None)
        if isinstance(c, Iteration):
            max_iters = c.max_iters if max_iters is None else min(max_iters, c.max_iters)
        elif isinstance(c, ResidualNorm):
            if res is not None:
                raise NotImplementedError("one residual criterion per solve on this path")
            res = c
        else:
            raise TypeError(f"unsupported criterion {c!r}")
    if max_iters is None:
        raise ValueError("an Iteration criterion is required")
    if res is None:
        return max_iters, 0.0, _BASELINES["rhs_norm"]
    return max_iters, res.reduction_factor, res.mode


# ---------------------------------------------------------- preconditioner --
class Jacobi:
    """Scalar Jacobi (preconditioner::Jacobi with max_block_size 1,
    core/preconditioner/jacobi.cpp:149-196, 337-369)."""

    @staticmethod
    def build():
        return _Builder(JacobiFactory, max_block_size=32)

    def __init__(self, A: Csr, aggregate_l1: bool = False):
        self.A = A
        self.aggregate_l1 = bool(aggregate_l1)
        self.inv_diag = torch.empty(A.shape[0], dtype=A.dtype, device=A.values.device)
        call(f"b2s_jacobi_invert_diagonal_{_SFX[A.dtype]}", A.shape[0],
             _p(A.row_ptrs), _p(A.col_idxs), _p(A.values), _p(self.inv_diag),
             int(self.aggregate_l1), _stream(self.inv_diag))

    def apply(self, *args):
        """apply(b, x) or apply(alpha, b, beta, x)."""
        if len(args) == 2:
            (b, x), alpha, beta = args, None, None
        else:
            a, b, be, x = args
            dev = self.A.values.device
            alpha = torch.as_tensor(a, dtype=self.A.dtype, device=dev).reshape(1)
            beta = torch.as_tensor(be, dtype=self.A.dtype, device=dev).reshape(1)
        b2 = _check_dense(b, self.A.shape[0], self.A.dtype, "b")
        x2 = _check_dense(x, self.A.shape[0], self.A.dtype, "x")
        call(f"b2s_jacobi_apply_{_SFX[self.A.dtype]}", b2.shape[0], b2.shape[1],
             _p(self.inv_diag), _p(b2), b2.stride(0), _p(x2), x2.stride(0),
             _p(alpha), _p(beta), _stream(x2))
        return x


def find_blocks(row_ptrs, col_idxs, max_block_size):
    """Block pointers of the diagonal blocks (jacobi::find_blocks,
    reference/preconditioner/jacobi_kernels.cpp:28-98): runs of consecutive
    rows with equal column patterns up to max_block_size rows (natural
    blocks), then neighbouring natural blocks merged while they fit.  Host
    set-up in the library (b2s_jacobi_find_blocks) on host Csr arrays."""
    rp = np.ascontiguousarray(row_ptrs, dtype=np.int32)
    ci = np.ascontiguousarray(col_idxs, dtype=np.int32)
    n = len(rp) - 1
    out = np.zeros(n + 1, dtype=np.int32)
    if len(ci) == 0:
        ci = np.zeros(1, dtype=np.int32)  # rows without entries: any valid buffer
    nb = call("b2s_jacobi_find_blocks", n, rp.ctypes.data, ci.ctypes.data,
              int(max_block_size), out.ctypes.data)
    return out[:nb + 1].copy()


# precision_reduction bytes, (preserving << 4) | non-preserving
# (include/ginkgo/core/base/types.hpp)
AUTODETECT = 0xFF


def precision_reduction(preserving: int, nonpreserving: int) -> int:
    """precision_reduction(preserving, nonpreserving) as its byte."""
    return (int(preserving) << 4) | int(nonpreserving)


class BlockJacobi:
    """preconditioner::Jacobi with max_block_size 2..32 (core/preconditioner/
    jacobi.cpp:370-420): the diagonal blocks inverted on the device
    (b2s_jacobi_block_generate_*), applied as x = D^-1 b or
    alpha D^-1 b + beta x.  The solvers apply the blocks inside their
    passes: CG in its update pass (b2s_cg_block_solve_*), BiCGStab to p' and
    s (b2s_bicgstab_block_solve_*), GMRES and IR over GMRES to each Krylov
    vector (b2s_gmres_block_solve).

    storage_optimization (Jacobi's parameter of that name): None or
    precision_reduction(0, 0) keeps full precision; one precision_reduction
    byte applies to every block, AUTODETECT choosing per block from its
    conditioning and `accuracy`; a sequence gives the blocks' requests in
    turn, repeated as needed (jacobi::initialize_precisions).  The blocks of
    a storage group share the most reduced precision all of them support
    (b2s_jacobi_block_generate_adaptive_*); `block_precisions` and
    `conditioning` hold the outcome.  The apply and the fused solvers read
    each group at its storage precision, widened to the value type."""

    def __init__(self, A: Csr, max_block_size: int, block_pointers=None,
                 aggregate_l1: bool = False, storage_optimization=None,
                 accuracy: float = 1e-1):
        self.A = A
        self.aggregate_l1 = bool(aggregate_l1)
        self.max_block_size = int(max_block_size)
        if not 1 <= self.max_block_size <= 32:
            raise ValueError("max_block_size must be 1..32")
        if block_pointers is None:
            block_pointers = find_blocks(A.row_ptrs.cpu().numpy(), A.col_idxs.cpu().numpy(),
                                         self.max_block_size)
        bp = np.asarray(block_pointers, dtype=np.int32)
        sizes = np.diff(bp)
        if bp[0] != 0 or bp[-1] != A.shape[0] or np.any(sizes < 0) or \
                np.any(sizes > self.max_block_size):
            raise ValueError("block pointers must run from 0 to num_rows in steps of "
                             "0..max_block_size")
        dev = A.values.device
        self.block_pointers = bp
        self.num_blocks = len(bp) - 1
        self._ptrs = torch.from_numpy(bp).to(dev)
        m = self.max_block_size
        bo, go, gp, space = C.c_int64(0), C.c_int64(0), C.c_int32(0), C.c_int64(0)
        call("b2s_jacobi_storage_scheme", m, self.num_blocks, C.byref(bo), C.byref(go),
             C.byref(gp), C.byref(space))
        # block_interleaved_storage_scheme: (block_offset, group_offset, group_power)
        self.storage_scheme = (int(bo.value), int(go.value), int(gp.value))
        self.blocks = torch.zeros(max(int(space.value), 1), dtype=A.dtype, device=dev)
        self.accuracy = float(accuracy)
        req = self._requests(storage_optimization)
        self._full = None
        if req is None:
            self._prec = None
            self.conditioning = None
            call(f"b2s_jacobi_block_generate_{_SFX[A.dtype]}", A.shape[0], _p(A.row_ptrs),
                 _p(A.col_idxs), _p(A.values), self.num_blocks, _p(self._ptrs), m,
                 _p(self.blocks), int(self.aggregate_l1), _stream(self.blocks))
            return
        self._prec = torch.from_numpy(req).to(dev)
        self.conditioning = torch.zeros(max(self.num_blocks, 1), dtype=A.dtype, device=dev)
        wb = C.c_int64(0)
        call("b2s_jacobi_adaptive_workspace_bytes", self.num_blocks, C.byref(wb))
        ws = torch.empty(max(int(wb.value), 4), dtype=torch.uint8, device=dev)
        acc = C.c_double(self.accuracy) if A.dtype == torch.float64 else C.c_float(self.accuracy)
        call(f"b2s_jacobi_block_generate_adaptive_{_SFX[A.dtype]}", A.shape[0],
             _p(A.row_ptrs), _p(A.col_idxs), _p(A.values), self.num_blocks, _p(self._ptrs), m,
             acc, _p(self.conditioning), _p(self._prec), _p(self.blocks),
             int(self.aggregate_l1), _p(ws), _stream(self.blocks))
        self.conditioning = self.conditioning[:self.num_blocks]

    def _requests(self, opt):
        """The per-block precision requests, or None for full precision."""
        if opt is None:
            return None
        if np.isscalar(opt):
            if int(opt) == 0:
                return None
            req = np.full(self.num_blocks, int(opt), dtype=np.uint8)
        else:
            src = np.asarray(opt, dtype=np.uint8).reshape(-1)
            if src.size == 0:
                raise ValueError("storage_optimization is an empty sequence")
            req = src[np.arange(self.num_blocks) % src.size]
        return np.ascontiguousarray(req) if req.size else np.zeros(1, np.uint8)

    @property
    def adaptive(self) -> bool:
        return self._prec is not None

    @property
    def block_precisions(self):
        """The storage precision of each block (precision_reduction bytes),
        or None for full precision."""
        return None if self._prec is None else self._prec[:self.num_blocks].cpu().numpy()

    @property
    def full_blocks(self):
        """The blocks at full precision in the interleaved layout (the
        storage itself, or its widened copy when adaptive)."""
        if self._prec is None:
            return self.blocks
        if self._full is None:
            self._full = torch.empty_like(self.blocks)
            call(f"b2s_jacobi_block_expand_{_SFX[self.A.dtype]}", self.num_blocks,
                 self.max_block_size, _p(self._prec), _p(self.blocks), _p(self._full),
                 _stream(self.blocks))
        return self._full

    @property
    def inv_diag(self):
        raise NotImplementedError("a block Jacobi preconditioner has no inverse "
                                  "diagonal; the solvers take its blocks")

    def apply(self, *args):
        """apply(b, x) or apply(alpha, b, beta, x)."""
        n = self.A.shape[0]
        if len(args) == 2:
            (b, x), alpha, beta = args, None, None
        else:
            a, b, be, x = args
            dev = self.A.values.device
            alpha = torch.as_tensor(a, dtype=self.A.dtype, device=dev).reshape(1)
            beta = torch.as_tensor(be, dtype=self.A.dtype, device=dev).reshape(1)
        b2 = _check_dense(b, n, self.A.dtype, "b")
        x2 = _check_dense(x, n, self.A.dtype, "x")
        if self._prec is None:
            call(f"b2s_jacobi_block_apply_{_SFX[self.A.dtype]}", n, self.num_blocks,
                 _p(self._ptrs), self.max_block_size, _p(self.blocks), _p(b2), b2.stride(0),
                 _p(x2), x2.stride(0), b2.shape[1], _p(alpha), _p(beta), _stream(x2))
        else:
            call(f"b2s_jacobi_block_apply_adaptive_{_SFX[self.A.dtype]}", n, self.num_blocks,
                 _p(self._ptrs), self.max_block_size, _p(self._prec), _p(self.blocks),
                 _p(b2), b2.stride(0), _p(x2), x2.stride(0), b2.shape[1], _p(alpha),
                 _p(beta), _stream(x2))
        return x

    def _positions(self):
        """Index of entry (i, j) of block b in the interleaved storage, as an
        array [num_blocks, m, m] (get_global_block_offset(b) + i + j * stride,
        include/ginkgo/core/preconditioner/jacobi.hpp:100-140)."""
        bo, go, gp = self.storage_scheme
        gs = 1 << gp
        stride = bo << gp
        m = self.max_block_size
        b = np.arange(self.num_blocks)[:, None, None]
        i = np.arange(m)[None, :, None]
        j = np.arange(m)[None, None, :]
        return (b >> gp) * go + (b & (gs - 1)) * bo + i + j * stride

    def block(self, b):
        """The max_block_size x max_block_size slot of block b (host, full
        precision)."""
        return self.full_blocks.cpu().numpy()[self._positions()[b]]

    def to_dense(self):
        """The block-diagonal inverse as a dense host array."""
        n = self.A.shape[0]
        blk = self.full_blocks.cpu().numpy()
        pos = self._positions()
        out = np.zeros((n, n), dtype=blk.dtype)
        for i, (s, e) in enumerate(zip(self.block_pointers[:-1], self.block_pointers[1:])):
            bs = e - s
            out[s:e, s:e] = blk[pos[i]][:bs, :bs]
        return out

    def transpose(self):
        """Jacobi::transpose: the same blocks, each transposed in place in
        the interleaved layout."""
        t = BlockJacobi.__new__(BlockJacobi)
        t.__dict__.update(self.__dict__)
        pos = self._positions()
        src = torch.from_numpy(pos.transpose(0, 2, 1).reshape(-1)).to(self.blocks.device)
        dst = torch.from_numpy(pos.reshape(-1)).to(self.blocks.device)
        full = self.full_blocks
        t.blocks = full.clone()
        if len(dst):
            t.blocks[dst] = full[src]
        t._full = None
        if self._prec is not None:
            # the transposed values are the stored ones: rounding them to the
            # same precisions is exact
            t._full = t.blocks.clone()
            call(f"b2s_jacobi_block_reduce_{_SFX[self.A.dtype]}", self.num_blocks,
                 self.max_block_size, _p(self._prec), _p(t._full), _p(t.blocks),
                 _stream(t.blocks))
        return t


class JacobiFactory:
    """Jacobi::build() parameters: max_block_size (1 scalar, 2..32 blocks),
    block_pointers, aggregate_l1, storage_optimization and accuracy
    (include/ginkgo/core/preconditioner/jacobi.hpp, parameters; accuracy
    defaults to 1e-1 as there)."""

    def __init__(self, exec_, max_block_size=32, block_pointers=None, aggregate_l1=False,
                 storage_optimization=None, accuracy=1e-1):
        self.max_block_size = int(max_block_size)
        self.block_pointers = block_pointers
        self.aggregate_l1 = bool(aggregate_l1)
        self.storage_optimization = storage_optimization
        self.accuracy = float(accuracy)

    def generate(self, A):
        if self.max_block_size == 1:
            return Jacobi(A, self.aggregate_l1)
        return BlockJacobi(A, self.max_block_size, self.block_pointers, self.aggregate_l1,
                           self.storage_optimization, self.accuracy)


# ---------------------------------------------------------------- logging --
@dataclass
class ConvergenceLog:
    """What gko::log::Convergence records for one apply."""
    num_iterations: int = 0
    residual_norm: list = field(default_factory=list)
    has_converged: bool = False
    status: list = field(default_factory=list)
    restarts: int = 0


# ----------------------------------------------------------------- solvers --
class _SolverFactory:
    kind = ""

    def __init__(self, exec_, criteria=(), preconditioner=None, krylov_dim=100,
                 check_every=8, storage_precision=None, inner_reduction=1e-6,
                 ortho_method="mgs"):
        self.exec = exec_
        crit = criteria if isinstance(criteria, (list, tuple)) else (criteria,)
        self.max_iters, self.reduction, self.residual_mode = _criteria(crit)
        self.preconditioner = preconditioner
        # 1..128: the device rejects anything else (no silent change)
        self.krylov_dim = int(krylov_dim)
        if ortho_method not in _ORTHO:
            raise ValueError(f"unknown ortho_method {ortho_method!r}: one of {sorted(_ORTHO)}")
        self.ortho_method = ortho_method
        self.check_every = int(check_every)
        self.storage_precision = storage_precision
        self.inner_reduction = float(inner_reduction)

    def generate(self, A: Csr):
        return _Solver(self, A)


class _Solver:
    def __init__(self, factory, A):
        self.f = factory
        self.A = A
        self.logger = ConvergenceLog()
        prec = factory.preconditioner
        if isinstance(prec, _Builder):
            prec = prec.on(factory.exec)
        self.precond = prec.generate(A) if prec is not None else None
        self._ws = None

    def _workspace(self, nbytes):
        if nbytes < 0:
            raise GinkgoError("workspace", -1, "unsupported size")
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8,
                                   device=self.A.values.device)
        return self._ws

    @property
    def inv_diag(self):
        return None if self.precond is None else self.precond.inv_diag

    def apply(self, b, x):
        kind = self.f.kind
        if kind in ("cg", "bicgstab"):
            return self._apply_cg(b, x)
        if kind in ("gmres", "ir", "cb_gmres"):
            return self._apply_gmres(b, x)
        raise NotImplementedError(kind)

    def _apply_cg(self, b, x):
        A = self.A
        n = A.shape[0]
        b2 = _check_dense(b, n, A.dtype, "b")
        x2 = _check_dense(x, n, A.dtype, "x")
        k = b2.shape[1]
        name = self.f.kind
        it = C.c_int64(0)
        res = np.zeros(k, np.float64)
        st = np.zeros(k, np.uint8)
        tail = (_p(b2), b2.stride(0), _p(x2), x2.stride(0), k, self.f.max_iters,
                self.f.reduction, self.f.residual_mode, self.f.check_every)
        outs = (C.byref(it), res.ctypes.data_as(C.c_void_p),
                st.ctypes.data_as(C.c_void_p), _stream(x2))
        M = self.precond
        if isinstance(M, BlockJacobi):
            nbytes = getattr(lib(), f"b2s_{name}_block_workspace_bytes")(
                n, k, A.values.element_size())
            ws = self._workspace(nbytes)
            call(f"b2s_{name}_block_solve_{_SFX[A.dtype]}", n, _p(A.row_ptrs),
                 _p(A.col_idxs), _p(A.values), A.max_row_nnz, M.num_blocks, _p(M._ptrs),
                 M.max_block_size, _p(M._prec), _p(M.blocks), *tail, _p(ws), ws.numel(),
                 *outs)
        else:
            nbytes = getattr(lib(), f"b2s_{name}_workspace_bytes")(
                n, k, A.values.element_size())
            ws = self._workspace(nbytes)
            call(f"b2s_{name}_solve_{_SFX[A.dtype]}", n, _p(A.row_ptrs), _p(A.col_idxs),
                 _p(A.values), A.max_row_nnz, _p(self.inv_diag), *tail, _p(ws), ws.numel(),
                 *outs)
        self.logger = ConvergenceLog(int(it.value), res.tolist(),
                                     bool(np.all(st & 0x80)), st.tolist())
        return x

    def _apply_gmres(self, b, x):
        A = self.A
        if A.dtype != torch.float64:
            raise TypeError("GMRES on this path takes the FP64 matrix; the "
                            "low-precision inner solve converts it itself")
        if self.f.residual_mode & _STOP_IMPLICIT:
            raise NotImplementedError("GMRES provides no implicit squared residual norm "
                                      "(the reference raises NotSupported too)")
        n = A.shape[0]
        b2 = _check_dense(b, n, A.dtype, "b")
        x2 = _check_dense(x, n, A.dtype, "x")
        k = b2.shape[1]
        if self.f.kind == "cb_gmres":
            sp = self.f.storage_precision or "reduce1"
            if sp not in _CB_STORAGE:
                raise ValueError(f"unknown CbGmres storage_precision {sp!r}: one of "
                                 f"{sorted(_CB_STORAGE)}")
            variant = _CB_STORAGE[sp]
        else:
            variant = {None: 0, "f64": 0, "f32": 1, "bf16": 2}[self.f.storage_precision]
        nbytes = lib().b2s_gmres_workspace_bytes(n, A.nnz, A.max_row_nnz, k,
                                                 self.f.krylov_dim, variant)
        if nbytes < 0:
            raise GinkgoError("b2s_gmres_workspace_bytes", -1,
                              f"krylov_dim {self.f.krylov_dim} is not supported: 1..128")
        ws = self._workspace(nbytes)
        it = np.zeros(k, np.int64)
        rs = np.zeros(k, np.int64)
        rn = np.zeros(k, np.float64)
        st = np.zeros(k, np.uint8)
        tail = (_p(b2), b2.stride(0), _p(x2), x2.stride(0), k, self.f.krylov_dim,
                self.f.max_iters, self.f.reduction, self.f.residual_mode,
                self.f.inner_reduction, _p(ws), ws.numel(), it.ctypes.data_as(C.c_void_p),
                rs.ctypes.data_as(C.c_void_p), rn.ctypes.data_as(C.c_void_p),
                st.ctypes.data_as(C.c_void_p), _stream(x2))
        M = self.precond
        if isinstance(M, BlockJacobi):
            call("b2s_gmres_block_solve", variant, _ORTHO[self.f.ortho_method], n,
                 _p(A.row_ptrs), _p(A.col_idxs), _p(A.values), A.max_row_nnz, M.num_blocks,
                 _p(M._ptrs), M.max_block_size, _p(M._prec), _p(M.blocks), *tail)
        else:
            call("b2s_gmres_solve", variant, _ORTHO[self.f.ortho_method], n,
                 _p(A.row_ptrs), _p(A.col_idxs), _p(A.values), A.max_row_nnz,
                 _p(self.inv_diag), *tail)
        self.logger = ConvergenceLog(int(it.max()) if k else 0, rn.tolist(),
                                     bool(np.all(st & 0x80)), st.tolist(),
                                     int(rs.max()) if k else 0)
        self.logger.iterations_per_column = it.tolist()
        return x


class _CgFactory(_SolverFactory):
    kind = "cg"


class _BicgstabFactory(_SolverFactory):
    kind = "bicgstab"


class _GmresFactory(_SolverFactory):
    kind = "gmres"


class _CbGmresFactory(_SolverFactory):
    kind = "cb_gmres"


class _IrFactory(_SolverFactory):
    kind = "ir"

    def __init__(self, exec_, criteria=(), solver=None, **kw):
        inner = solver.params() if isinstance(solver, _Builder) else dict(solver or {})
        sp = inner.get("storage_precision", "f32")
        super().__init__(exec_, criteria=criteria,
                         preconditioner=inner.get("preconditioner", kw.pop("preconditioner", None)),
                         krylov_dim=inner.get("krylov_dim", 100),
                         ortho_method=inner.get("ortho_method", "mgs"),
                         storage_precision=sp if sp != "f64" else "f32",
                         inner_reduction=inner.get("inner_reduction", 1e-6), **kw)


class Cg:
    """solver::Cg (core/solver/cg.cpp)."""

    @staticmethod
    def build():
        return _Builder(_CgFactory)


class Bicgstab:
    """solver::Bicgstab (core/solver/bicgstab.cpp)."""

    @staticmethod
    def build():
        return _Builder(_BicgstabFactory)


class Gmres:
    """solver::Gmres (core/solver/gmres.cpp): krylov_dim 1..128 (default
    100, as the reference), ortho_method "mgs" (default; run as CGS2 on the
    device), "cgs" or "cgs2", any number of right-hand sides (independent
    columns).  with_storage_precision("f32" or "bf16") selects the
    low-precision Arnoldi used inside Ir."""

    @staticmethod
    def build():
        return _Builder(_GmresFactory, krylov_dim=100)


class CbGmres:
    """solver::CbGmres (core/solver/cb_gmres.cpp): restarted GMRES with FP64
    arithmetic and the Krylov basis stored in a reduced format,
    with_storage_precision: "keep" (FP64), "reduce1" (FP32, the default),
    "reduce2" (half), "integer" (int64), "ireduce1" (int32), "ireduce2"
    (int16), the integers with one scale per vector.  krylov_dim 1..128
    (default 100, as the reference)."""

    @staticmethod
    def build():
        return _Builder(_CbGmresFactory, krylov_dim=100, storage_precision="reduce1")


class Ir:
    """solver::Ir (core/solver/ir.cpp) with a low-precision GMRES cycle as
    the inner solver and the FP64 residual outside."""

    @staticmethod
    def build():
        return _Builder(_IrFactory)
