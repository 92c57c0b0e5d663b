"""Batched solve over many independent systems of uneven size, named after
the reference's ``gko::batch::matrix::Ell`` and
``gko::batch::solver::Bicgstab``:

    A = BatchEll.from_csr(exec, systems)          # list of (rp, ci, v)
    solver = (BatchBicgstab.build().with_max_iterations(500)
              .with_tolerance(1e-8).with_tolerance_type("relative")
              .with_preconditioner("jacobi").on(exec).generate(A))
    solver.apply(b, x)        # b, x: concatenated per-system vectors
    solver.logger.iterations  # per system, as batch::log::BatchConvergence

The reference's batches are uniform (one size, shared column indices); this
batch is ragged: every system has its own size and pattern.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import stencils
from ._lib import call, lib
from .matrix import _p, _stream

_SFX = {torch.float64: "f64", torch.float32: "f32"}


class BatchEll:
    """Ragged batch Ell: system s owns rows [row_offsets[s], row_offsets[s+1])
    and its entries at values[width * row_offsets[s] + j * n_s + r].
    BatchEll.uniform builds the reference's own uniform batch::matrix::Ell
    (one size, one column-index array shared by all systems)."""

    uniform_rows = None  # rows per system when the column indices are shared

    def __init__(self, exec_, row_offsets, width, col_idxs, values):
        dev = exec_.device
        self.exec = exec_
        self.host_row_offsets = np.ascontiguousarray(row_offsets, dtype=np.int32)
        self.row_offsets = torch.from_numpy(self.host_row_offsets).to(dev)
        self.width = int(width)
        self.col_idxs = torch.as_tensor(col_idxs, dtype=torch.int32).to(dev).contiguous()
        self.values = torch.as_tensor(values).to(dev).contiguous()
        self.dtype = self.values.dtype
        self.num_systems = len(self.host_row_offsets) - 1
        self.total_rows = int(self.host_row_offsets[-1])

    @property
    def sizes(self):
        return np.diff(self.host_row_offsets)

    @classmethod
    def uniform(cls, exec_, num_systems, num_rows, width, col_idxs, values):
        """batch::matrix::Ell (include/ginkgo/core/matrix/batch_ell.hpp):
        num_systems systems of num_rows rows, col_idxs (num_rows * width,
        column-major, -1 = padding) shared by all systems, values
        (num_systems * num_rows * width) per system."""
        offs = np.arange(num_systems + 1, dtype=np.int64) * num_rows
        A = cls(exec_, offs, width, col_idxs, values)
        if A.col_idxs.numel() != num_rows * width:
            raise ValueError("shared col_idxs must hold num_rows * width entries")
        if A.values.numel() != num_systems * num_rows * width:
            raise ValueError("values must hold num_systems * num_rows * width entries")
        A.uniform_rows = int(num_rows)
        return A

    @classmethod
    def from_csr(cls, exec_, systems, width=None, dtype=torch.float64):
        """systems: list of (row_ptrs, col_idxs, values), local indices."""
        sizes = np.array([len(rp) - 1 for rp, _, _ in systems], dtype=np.int64)
        offs = np.zeros(len(systems) + 1, dtype=np.int64)
        np.cumsum(sizes, out=offs[1:])
        if width is None:
            width = max(int(np.diff(rp).max()) if len(rp) > 1 else 0
                        for rp, _, _ in systems)
        ci = np.full(int(offs[-1]) * width, -1, dtype=np.int32)
        v = np.zeros(int(offs[-1]) * width, dtype=np.float64)
        for s, (rp, c, val) in enumerate(systems):
            n = len(rp) - 1
            rp = np.asarray(rp)
            lens = np.diff(rp)
            rows = np.repeat(np.arange(n), lens)
            slot = np.arange(len(c)) - np.repeat(rp[:-1], lens)
            idx = width * offs[s] + slot * n + rows
            ci[idx] = c
            v[idx] = val
        return cls(exec_, offs, width, torch.from_numpy(ci),
                   torch.from_numpy(v).to(dtype))

    def to_csr_list(self):
        """Host CSR per system (for checking)."""
        ci = self.col_idxs.cpu().numpy()
        if self.uniform_rows is not None:
            ci = np.tile(ci, self.num_systems)
        v = self.values.cpu().numpy()
        out = []
        for s in range(self.num_systems):
            o, n = int(self.host_row_offsets[s]), int(self.sizes[s])
            base = self.width * o
            rows, cols, vals = [], [], []
            for j in range(self.width):
                c = ci[base + j * n: base + (j + 1) * n]
                m = c >= 0
                rows.append(np.nonzero(m)[0])
                cols.append(c[m])
                vals.append(v[base + j * n: base + (j + 1) * n][m])
            rows, cols, vals = map(np.concatenate, (rows, cols, vals))
            order = np.lexsort((cols, rows))
            rp = np.zeros(n + 1, dtype=np.int64)
            np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
            out.append((rp.astype(np.int32), cols[order], vals[order]))
        return out


def convection_diffusion_batch(exec_, num_systems, lo=32, hi=1024, seed=0,
                               dtype=torch.float64):
    """The batched workload: system sizes ~ U[lo, hi]; each system a 5-point
    convection-diffusion stencil on the most-square grid with nx * ny = n,
    diffusion ~ U[0.5, 2], velocity components ~ U[-1, 1] (central
    differences, unit mesh width)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=num_systems)
    diff = rng.uniform(0.5, 2.0, size=num_systems)
    vel = rng.uniform(-1.0, 1.0, size=(num_systems, 2))
    systems = []
    cache = {}
    for s in range(num_systems):
        n = int(sizes[s])
        nx, ny = stencils.most_square_grid(n)
        key = (nx, ny)
        if key not in cache:
            cache[key] = stencils.convection_diffusion_2d(nx, ny, 1.0, 0.0, 0.0)
        rp, ci, _ = cache[key]
        # weights of the pattern: diag, east, west, north, south
        d = diff[s]
        vx, vy = vel[s]
        rows = np.repeat(np.arange(n), np.diff(rp))
        off = ci.astype(np.int64) - rows
        w = np.where(off == 0, 4 * d,
            np.where(off == 1, -d + 0.5 * vx,
            np.where(off == -1, -d - 0.5 * vx,
            np.where(off == nx, -d + 0.5 * vy, -d - 0.5 * vy))))
        systems.append((rp, ci, w))
    return BatchEll.from_csr(exec_, systems, width=5, dtype=dtype), systems


class _Builder:
    def __init__(self):
        self.p = {"max_iterations": 100, "tolerance": 1e-11,
                  "tolerance_type": "absolute", "preconditioner": None}

    def __getattr__(self, name):
        if name.startswith("with_"):
            def setter(v):
                self.p[name[5:]] = v
                return self
            return setter
        raise AttributeError(name)

    def on(self, exec_):
        return _BatchFactory(exec_, dict(self.p))


class _BatchFactory:
    def __init__(self, exec_, params):
        self.exec = exec_
        self.p = params

    def generate(self, A: BatchEll):
        return _BatchSolver(self, A)


class BatchLog:
    def __init__(self, iterations, residual_norms):
        self.iterations = iterations
        self.residual_norms = residual_norms


class _BatchSolver:
    def __init__(self, f, A):
        self.f = f
        self.A = A
        self.tune_table = None
        dev = A.values.device
        self.iters = torch.zeros(A.num_systems, dtype=torch.int32, device=dev)
        self.res = torch.zeros(A.num_systems, dtype=torch.float64, device=dev)
        nbytes = lib().b2s_batch_bicgstab_workspace_bytes(
            A.num_systems, A.total_rows, A.values.element_size())
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.logger = None

    def _args(self, b, x):
        A, p = self.A, self.f.p
        for t, nm in ((b, "b"), (x, "x")):
            if t.dtype != A.dtype or t.numel() != A.total_rows or not t.is_contiguous():
                raise ValueError(f"{nm} must be a contiguous {A.dtype} vector of "
                                 f"{A.total_rows} entries")
        tol_abs = 1 if p["tolerance_type"] == "absolute" else 0
        jac = 1 if p["preconditioner"] in ("jacobi", "scalar_jacobi") else 0
        return (A.num_systems, _p(A.row_offsets),
                A.host_row_offsets.ctypes.data_as(C.c_void_p), A.width,
                _p(A.col_idxs), _p(A.values), _p(b), _p(x),
                int(p["max_iterations"]), float(p["tolerance"]), tol_abs, jac)

    def _uniform_call(self, b, x, tt, table_out):
        A = self.A
        args = self._args(b, x)  # validates b and x
        call(f"b2s_batch_ell_uniform_bicgstab_solve_{_SFX[A.dtype]}", A.num_systems,
             A.uniform_rows, A.width, _p(A.col_idxs), _p(A.values), _p(b), _p(x),
             *args[8:], tt, _p(self.ws), self.ws.numel(), _p(self.iters), _p(self.res),
             _stream(x), table_out)

    def apply(self, b, x):
        tt = None if self.tune_table is None else \
            self.tune_table.ctypes.data_as(C.c_void_p)
        if self.A.uniform_rows is not None:
            self._uniform_call(b, x, tt, None)
        else:
            call(f"b2s_batch_ell_bicgstab_solve_{_SFX[self.A.dtype]}",
                 *self._args(b, x), tt, _p(self.ws), self.ws.numel(),
                 _p(self.iters), _p(self.res), _stream(x))
        self.logger = BatchLog(self.iters, self.res)
        return x

    def tune(self, b, x):
        """Autotunes threads-per-system and vector placement per size bucket
        (and solves); later applies reuse the table."""
        table = np.zeros(24, dtype=np.int32)
        if self.A.uniform_rows is not None:
            self._uniform_call(b, x, None, table.ctypes.data_as(C.c_void_p))
        else:
            call(f"b2s_batch_ell_bicgstab_tune_{_SFX[self.A.dtype]}",
                 *self._args(b, x), _p(self.ws), self.ws.numel(), _p(self.iters),
                 _p(self.res), table.ctypes.data_as(C.c_void_p), _stream(x))
        self.tune_table = table
        self.logger = BatchLog(self.iters, self.res)
        return table


class BatchBicgstab:
    """batch::solver::Bicgstab (core/solver/batch_bicgstab.cpp)."""

    @staticmethod
    def build():
        return _Builder()


# --------------------------------------------------------- multi-GPU ------

def shard_bounds(row_offsets, world: int) -> np.ndarray:
    """Split of the systems into `world` contiguous shards of about equal
    rows (the work of an iteration is proportional to rows): rank k owns
    systems [bounds[k], bounds[k + 1]).  Each shard's rows are within one
    system of total / world; ranks beyond the number of systems get none."""
    offs = np.asarray(row_offsets, dtype=np.int64)
    total = int(offs[-1])
    targets = np.array([total * k / world for k in range(world + 1)])
    bounds = np.searchsorted(offs, targets, side="left").astype(np.int64)
    bounds[0], bounds[-1] = 0, len(offs) - 1
    return np.maximum.accumulate(bounds)


def slice_systems(A: BatchEll, s0: int, s1: int, exec_) -> BatchEll:
    """Systems [s0, s1) of A as a batch on exec_ (their storage is one
    contiguous slice: system s owns entries from width * row_offsets[s])."""
    o0, o1 = int(A.host_row_offsets[s0]), int(A.host_row_offsets[s1])
    w = A.width
    if A.uniform_rows is not None:
        return BatchEll.uniform(exec_, s1 - s0, A.uniform_rows, w, A.col_idxs,
                                A.values[w * o0:w * o1])
    return BatchEll(exec_, A.host_row_offsets[s0:s1 + 1] - o0, w,
                    A.col_idxs[w * o0:w * o1], A.values[w * o0:w * o1])


def _all_gather_segments(local, lengths, group):
    """Concatenation over ranks of each rank's 1-D segment (lengths known on
    every rank): one all-gather of segments padded to the longest."""
    import torch.distributed as dist
    world = len(lengths)
    m = max(int(n) for n in lengths)
    if m == 0:
        return local[:0]
    pad = torch.zeros(m, dtype=local.dtype, device=local.device)
    pad[:local.numel()] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:int(n)] for p, n in zip(parts, lengths)])


def solve_sharded(A: BatchEll, b, x, exec_, factory=None, group=None, local_solve=None):
    """Solves the independent systems of A across the ranks of `group` (the
    default process group when None): rank k solves its contiguous shard
    (shard_bounds) on exec_, its own device, and every rank receives the
    whole solution, the iteration counts and the residual norms through one
    all-gather each; there is no other communication.  A, b and x hold the
    whole batch (host or device); x is overwritten with the solution.
    factory: a BatchBicgstab builder (the .build()....with_*() chain), used
    on exec_; local_solve(A_local, b_local, x_local) -> (x, iterations,
    residual_norms) replaces it (a host solver in tests).  Returns
    (x, iterations, residual_norms)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bounds = shard_bounds(A.host_row_offsets, world)
    s0, s1 = int(bounds[rank]), int(bounds[rank + 1])
    offs = A.host_row_offsets
    o0, o1 = int(offs[s0]), int(offs[s1])
    A_loc = slice_systems(A, s0, s1, exec_)
    dev = exec_.device
    b_loc = b[o0:o1].to(dev).contiguous()
    x_loc = x[o0:o1].to(dev).contiguous()
    if local_solve is None:
        if s1 > s0:
            solver = factory.on(exec_).generate(A_loc)
            solver.apply(b_loc, x_loc)
            iters, res = solver.logger.iterations, solver.logger.residual_norms
        else:
            iters = torch.zeros(0, dtype=torch.int32, device=dev)
            res = torch.zeros(0, dtype=torch.float64, device=dev)
    else:
        x_loc, iters, res = local_solve(A_loc, b_loc, x_loc)
    row_len = [int(offs[bounds[k + 1]] - offs[bounds[k]]) for k in range(world)]
    sys_len = [int(bounds[k + 1] - bounds[k]) for k in range(world)]
    x_all = _all_gather_segments(x_loc.reshape(-1), row_len, group)
    it_all = _all_gather_segments(iters.to(dev, torch.int64).reshape(-1), sys_len, group)
    res_all = _all_gather_segments(res.to(dev, torch.float64).reshape(-1), sys_len, group)
    x.copy_(x_all.to(x.device))
    return x, it_all, res_all
