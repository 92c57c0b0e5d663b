"""Host-side matrix formats over the C ABI, named after the reference's
``gko::matrix`` classes (Csr, Ell, Sellp) and ``gko::CudaExecutor``.

Device storage is torch tensors (torch is used for memory, streams and the
autograd entry point only).  Dense operands are torch tensors of shape (n,)
or (n, k), row-major; ``apply(b, x)`` computes x = A b and
``apply(alpha, b, beta, x)`` computes x = alpha A b + beta x, as
``gko::LinOp::apply`` does (include/ginkgo/core/base/lin_op.hpp:129-203).
Every kernel launches on the current torch CUDA stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import call, lib

_SFX = {torch.float64: "f64", torch.float32: "f32"}
# B2S_VALUE_* codes of the mixed-type entry points
_VT = {torch.float64: 0, torch.float32: 1}


class CudaExecutor:
    """One device; kernels go to torch's current stream on that device
    (the reference's CudaExecutor owns one stream, executor.hpp:1723)."""

    def __init__(self, device_id: int = 0):
        self.device = torch.device("cuda", device_id)

    @staticmethod
    def create(device_id: int = 0):
        return CudaExecutor(device_id)

    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def synchronize(self):
        torch.cuda.synchronize(self.device)


def _stream(t: torch.Tensor):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _as2d(t: torch.Tensor):
    return t.unsqueeze(1) if t.dim() == 1 else t


def _check_dense(t: torch.Tensor, rows: int, dtype, what: str):
    """dtype None accepts FP64 and FP32 (mixed-precision operands)."""
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor")
    if dtype is None:
        if t.dtype not in _SFX:
            raise TypeError(f"{what} has dtype {t.dtype}, expected float64 or float32")
    elif t.dtype != dtype:
        raise TypeError(f"{what} has dtype {t.dtype}, expected {dtype}")
    t2 = _as2d(t)
    if t2.shape[0] != rows:
        raise ValueError(f"{what} has {t2.shape[0]} rows, expected {rows} "
                         "(DimensionMismatch)")
    if t2.dim() != 2 or t2.stride(1) != 1:
        raise ValueError(f"{what} must be row-major with unit column stride")
    return t2


def _scalar(v, dtype, device):
    if v is None:
        return None
    if isinstance(v, torch.Tensor):
        return v.to(device=device, dtype=dtype).reshape(1)
    return torch.tensor([v], dtype=dtype, device=device)


class _SparseBase:
    dtype: torch.dtype
    shape: tuple

    def _apply_args(self, args, mixed=False):
        """(b, x, alpha, beta) as 2-D views; with mixed, b and x may each be
        FP64 or FP32 (alpha then has the matrix type, beta the type of x, as
        core/matrix/csr.cpp:301-311 converts them)."""
        if len(args) == 2:
            b, x = args
            alpha = beta = None
        elif len(args) == 4:
            alpha, b, beta, x = args
        else:
            raise TypeError("apply(b, x) or apply(alpha, b, beta, x)")
        n, m = self.shape
        b2 = _check_dense(b, m, None if mixed else self.dtype, "b")
        x2 = _check_dense(x, n, None if mixed else self.dtype, "x")
        if b2.shape[1] != x2.shape[1]:
            raise ValueError("b and x have different numbers of columns")
        dev = x2.device
        return (b2, x2, _scalar(alpha, self.dtype, dev),
                _scalar(beta, x2.dtype, dev))

    def _uniform(self, b2, x2):
        return b2.dtype == self.dtype and x2.dtype == self.dtype


class Csr(_SparseBase):
    """Compressed sparse row matrix (int32 indices, float64/float32 values).

    strategy: "classical" (subwarp per row) or "load_balance" (merge-path
    tiles), the two strategies of include/ginkgo/core/matrix/csr.hpp:176-699.
    """

    def __init__(self, exec_, shape, row_ptrs, col_idxs, values,
                 strategy: str = "classical"):
        self.exec = exec_
        dev = exec_.device
        self.shape = (int(shape[0]), int(shape[1]))
        self.row_ptrs = torch.as_tensor(row_ptrs, dtype=torch.int32, device=dev).contiguous()
        self.col_idxs = torch.as_tensor(col_idxs, dtype=torch.int32, device=dev).contiguous()
        vals = torch.as_tensor(values, device=dev)
        if vals.dtype not in _SFX:
            vals = vals.to(torch.float64)
        self.values = vals.contiguous()
        self.dtype = self.values.dtype
        if self.row_ptrs.numel() != self.shape[0] + 1:
            raise ValueError("row_ptrs must have num_rows + 1 entries")
        self.nnz = int(self.col_idxs.numel())
        self._max_row_nnz = None
        self._tiles = None
        self.set_strategy(strategy)

    @classmethod
    def read(cls, exec_, rp, ci, v, shape=None, strategy="classical",
             dtype=torch.float64):
        rp = np.asarray(rp)
        n = len(rp) - 1
        shape = (n, n) if shape is None else shape
        vals = torch.as_tensor(np.asarray(v)).to(dtype)
        return cls(exec_, shape, torch.from_numpy(np.asarray(rp, np.int32)),
                   torch.from_numpy(np.asarray(ci, np.int32)), vals, strategy)

    def set_strategy(self, strategy: str):
        if strategy not in ("classical", "load_balance"):
            raise ValueError(f"unknown Csr strategy {strategy!r}")
        self.strategy = strategy
        if strategy == "load_balance" and self._tiles is None:
            nt = lib().b2s_csr_load_balance_num_tiles(self.shape[0], self.nnz)
            self._tiles = torch.empty(nt + 1, dtype=torch.int32,
                                      device=self.values.device)
            call("b2s_csr_load_balance_setup", self.shape[0], self.nnz,
                 _p(self.row_ptrs), nt, _p(self._tiles), _stream(self.values))
        return self

    @property
    def max_row_nnz(self) -> int:
        if self._max_row_nnz is None:
            ws = torch.empty(1, dtype=torch.int64, device=self.values.device)
            out = C.c_int64(0)
            call("b2s_csr_max_row_nnz", self.shape[0], _p(self.row_ptrs),
                 C.byref(out), _p(ws), _stream(self.values))
            self._max_row_nnz = int(out.value)
        return self._max_row_nnz

    def apply(self, *args):
        """x = A b or x = alpha A b + beta x; b and x may each be FP64 or
        FP32 (mixed types run in the most precise of the three).  As in the
        reference (core/matrix/csr.cpp:257-314): with b a Csr matrix and x a
        Csr, x = A b (SpGEMM) or x = alpha A b + beta x; with b an Identity,
        x = alpha A + beta x (SpGEAM).  x's arrays are replaced."""
        b = args[1] if len(args) == 4 else args[0]
        if isinstance(b, (Csr, Identity)):
            return self._apply_sparse(args)
        b2, x2, alpha, beta = self._apply_args(args, mixed=True)
        if not self._uniform(b2, x2):
            call("b2s_csr_spmv_mixed", _VT[self.dtype], _VT[b2.dtype], _VT[x2.dtype],
                 self.shape[0], self.shape[1], _p(self.row_ptrs), _p(self.col_idxs),
                 _p(self.values), self.max_row_nnz, _p(b2), b2.stride(0), _p(x2),
                 x2.stride(0), x2.shape[1], _p(alpha), _p(beta), _stream(x2))
            return args[-1]
        strat = 1 if self.strategy == "load_balance" else 0
        nt = 0 if self._tiles is None else self._tiles.numel() - 1
        call(f"b2s_csr_spmv_{_SFX[self.dtype]}", strat, self.shape[0],
             self.shape[1], _p(self.row_ptrs), _p(self.col_idxs),
             _p(self.values), self.max_row_nnz if strat == 0 else 0,
             _p(self._tiles), nt, _p(b2), b2.stride(0), _p(x2), x2.stride(0),
             x2.shape[1], _p(alpha), _p(beta), _stream(x2))
        return args[-1]

    def _apply_sparse(self, args):
        if len(args) == 2:
            b, x = args
            if isinstance(b, Identity):
                raise TypeError("A.apply(Identity, x): use apply(alpha, Identity, beta, x)")
            x._replace(spgemm(self, b))
        else:
            alpha, b, beta, x = args
            if not isinstance(x, Csr):
                raise TypeError("the result of a sparse product is a Csr matrix")
            if isinstance(b, Identity):
                x._replace(spgeam(alpha, self, beta, x))
            else:
                x._replace(spgemm(self, b, alpha=alpha, beta=beta, d=x))
        return args[-1]

    def _replace(self, other):
        """Takes other's arrays (the result of a sparse product)."""
        self.shape, self.row_ptrs, self.col_idxs = other.shape, other.row_ptrs, other.col_idxs
        self.values, self.dtype, self.nnz = other.values, other.dtype, other.nnz
        self._max_row_nnz, self._tiles = None, None
        self.set_strategy(self.strategy)

    def convert_to_hybrid(self, strategy="automatic", **params):
        """Csr -> Hybrid with one of the reference's width strategies
        (hybrid_config): the Ell width and Coo size are set up on the host,
        the scatter runs on the device (b2s_csr_convert_to_hybrid_*)."""
        rp = self.row_ptrs.cpu().numpy().astype(np.int64)
        width, coo = hybrid_config(np.diff(rp), strategy,
                                   value_bytes=self.values.element_size(), **params)
        n = self.shape[0]
        dev = self.values.device
        ell_ci = torch.empty(max(width * n, 1), dtype=torch.int32, device=dev)
        ell_v = torch.empty(max(width * n, 1), dtype=self.dtype, device=dev)
        coo_r = torch.empty(max(coo, 1), dtype=torch.int32, device=dev)
        coo_c = torch.empty(max(coo, 1), dtype=torch.int32, device=dev)
        coo_v = torch.empty(max(coo, 1), dtype=self.dtype, device=dev)
        wsb = lib().b2s_hybrid_convert_workspace_bytes(n)
        ws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)
        call(f"b2s_csr_convert_to_hybrid_{_SFX[self.dtype]}", n, _p(self.row_ptrs),
             _p(self.col_idxs), _p(self.values), width, n, _p(ell_ci), _p(ell_v), coo,
             _p(coo_r), _p(coo_c), _p(coo_v), _p(ws), wsb, _stream(ell_v))
        return Hybrid(self.exec, self.shape, width, n, ell_ci[:width * n], ell_v[:width * n],
                      coo_r[:coo], coo_c[:coo], coo_v[:coo])

    def convert_to_precision(self, dtype):
        return Csr(self.exec, self.shape, self.row_ptrs, self.col_idxs,
                   self.values.to(dtype), self.strategy)

    def convert_to_ell(self, stride=None):
        n = self.shape[0]
        width = self.max_row_nnz
        stride = n if stride is None else int(stride)
        dev = self.values.device
        ci = torch.empty(width * stride, dtype=torch.int32, device=dev)
        v = torch.empty(width * stride, dtype=self.dtype, device=dev)
        call(f"b2s_csr_convert_to_ell_{_SFX[self.dtype]}", n, _p(self.row_ptrs),
             _p(self.col_idxs), _p(self.values), width, stride, _p(ci), _p(v),
             _stream(v))
        return Ell(self.exec, self.shape, width, stride, ci, v)

    def convert_to_sellp(self, slice_size: int = 64, stride_factor: int = 1):
        n = self.shape[0]
        dev = self.values.device
        ns = (n + slice_size - 1) // slice_size
        sets = torch.empty(ns + 1, dtype=torch.int64, device=dev)
        lens = torch.empty(max(ns, 1), dtype=torch.int64, device=dev)
        wsb = lib().b2s_sellp_slice_sets_workspace_bytes(n, slice_size)
        ws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)
        call("b2s_sellp_compute_slice_sets", n, _p(self.row_ptrs), slice_size,
             stride_factor, _p(sets), _p(lens), _p(ws), wsb, _stream(sets))
        total = int(sets[-1].item()) * slice_size  # host read, as csr.cpp:473
        # slots of the rows past num_rows in the last slice are never
        # written by the conversion; they hold padding (-1, 0)
        ci = torch.full((max(total, 1),), -1, dtype=torch.int32, device=dev)
        v = torch.zeros(max(total, 1), dtype=self.dtype, device=dev)
        call(f"b2s_csr_convert_to_sellp_{_SFX[self.dtype]}", n,
             _p(self.row_ptrs), _p(self.col_idxs), _p(self.values), slice_size,
             _p(sets), _p(lens), _p(ci), _p(v), _stream(v))
        return Sellp(self.exec, self.shape, slice_size, stride_factor, sets,
                     lens[:ns], ci[:total], v[:total])

    def transpose(self):
        n, m = self.shape
        dev = self.values.device
        wsb = lib().b2s_csr_transpose_workspace_bytes(
            n, m, self.nnz, self.values.element_size())
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        trp = torch.empty(m + 1, dtype=torch.int32, device=dev)
        tci = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        tv = torch.empty(max(self.nnz, 1), dtype=self.dtype, device=dev)
        call(f"b2s_csr_transpose_{_SFX[self.dtype]}", n, m, self.nnz,
             _p(self.row_ptrs), _p(self.col_idxs), _p(self.values), _p(trp),
             _p(tci), _p(tv), _p(ws), wsb, _stream(tv))
        return Csr(self.exec, (m, n), trp, tci[:self.nnz], tv[:self.nnz],
                   self.strategy)


class Ell(_SparseBase):
    """Column-major padded Ell (include/ginkgo/core/matrix/ell.hpp)."""

    def __init__(self, exec_, shape, width, stride, col_idxs, values):
        self.exec = exec_
        self.shape = tuple(shape)
        self.width, self.stride = int(width), int(stride)
        self.col_idxs, self.values = col_idxs, values
        self.dtype = values.dtype

    def apply(self, *args):
        """As Csr.apply: b and x may each be FP64 or FP32."""
        b2, x2, alpha, beta = self._apply_args(args, mixed=True)
        if not self._uniform(b2, x2):
            call("b2s_ell_spmv_mixed", _VT[self.dtype], _VT[b2.dtype], _VT[x2.dtype],
                 self.shape[0], self.shape[1], self.width, self.stride,
                 _p(self.col_idxs), _p(self.values), _p(b2), b2.stride(0), _p(x2),
                 x2.stride(0), x2.shape[1], _p(alpha), _p(beta), _stream(x2))
            return args[-1]
        call(f"b2s_ell_spmv_{_SFX[self.dtype]}", self.shape[0], self.shape[1],
             self.width, self.stride, _p(self.col_idxs), _p(self.values),
             _p(b2), b2.stride(0), _p(x2), x2.stride(0), x2.shape[1],
             _p(alpha), _p(beta), _stream(x2))
        return args[-1]


class Sellp(_SparseBase):
    """Sliced Ellpack (include/ginkgo/core/matrix/sellp.hpp); slice_sets and
    slice_lengths are uint64 on the device (held as int64 tensors)."""

    def __init__(self, exec_, shape, slice_size, stride_factor, slice_sets,
                 slice_lengths, col_idxs, values):
        self.exec = exec_
        self.shape = tuple(shape)
        self.slice_size, self.stride_factor = int(slice_size), int(stride_factor)
        self.slice_sets, self.slice_lengths = slice_sets, slice_lengths
        self.col_idxs, self.values = col_idxs, values
        self.dtype = values.dtype
        # the longest slice, for the SpMV's choice of one or two rows per
        # lane slot (read back once here)
        self.max_slice_length = int(slice_lengths.max().item()) if slice_lengths.numel() else 0

    @property
    def num_stored_elements(self):
        return int(self.values.numel())

    def apply(self, *args):
        """Operands of another type are converted to the matrix type and the
        result back (precision_dispatch, core/matrix/sellp.cpp:150-180)."""
        b2, x2, alpha, beta = self._apply_args(args, mixed=True)
        bt, xt = b2, x2
        if b2.dtype != self.dtype:
            bt = _convert(b2, self.dtype)
        if x2.dtype != self.dtype:
            xt = _convert(x2, self.dtype) if beta is not None else \
                torch.empty(x2.shape, dtype=self.dtype, device=x2.device)
            beta = None if beta is None else beta.to(self.dtype)
        call(f"b2s_sellp_spmv_hinted_{_SFX[self.dtype]}", self.shape[0], self.shape[1],
             self.slice_size, _p(self.slice_sets), _p(self.slice_lengths),
             _p(self.col_idxs), _p(self.values), _p(bt), bt.stride(0), _p(xt),
             xt.stride(0), xt.shape[1], _p(alpha), _p(beta), self.max_slice_length,
             _stream(xt))
        if xt is not x2:
            call("b2s_dense_convert", _VT[xt.dtype], _VT[x2.dtype], x2.shape[0], x2.shape[1],
                 _p(xt), xt.stride(0), _p(x2), x2.stride(0), _stream(x2))
        return args[-1]


class Identity:
    """matrix::Identity of size n: A.apply(alpha, Identity(n), beta, C)
    computes C = alpha A + beta C (SpGEAM), as the reference does."""

    def __init__(self, n):
        self.shape = (int(n), int(n))


def _dev_scalar(v, dtype, device):
    if v is None:
        return None
    return _scalar(v, dtype, device)


def spgemm(a: Csr, b: Csr, alpha=None, beta=None, d: Csr = None) -> Csr:
    """C = A B, or C = alpha A B + beta D (csr::spgemm / advanced_spgemm):
    bit-exact with the reference executor, columns ascending."""
    if a.shape[1] != b.shape[0]:
        raise ValueError("A's columns and B's rows differ (DimensionMismatch)")
    if a.dtype != b.dtype or (d is not None and d.dtype != a.dtype):
        raise TypeError("SpGEMM operands must share one value type")
    if (d is None) != (beta is None):
        raise ValueError("D and beta go together")
    if d is not None and d.shape != (a.shape[0], b.shape[1]):
        raise ValueError("D has the wrong shape (DimensionMismatch)")
    n, m = a.shape[0], b.shape[1]
    dev = a.values.device
    wsb = lib().b2s_csr_spgemm_workspace_bytes(n, m)
    ws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)
    rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    nnz = C.c_int64(0)
    st = _stream(a.values)
    call("b2s_csr_spgemm_symbolic", n, m, _p(a.row_ptrs), _p(a.col_idxs), _p(b.row_ptrs),
         _p(b.col_idxs), _p(d.row_ptrs) if d is not None else None,
         _p(d.col_idxs) if d is not None else None, _p(rp), C.byref(nnz), _p(ws), wsb, st)
    k = int(nnz.value)
    ci = torch.empty(max(k, 1), dtype=torch.int32, device=dev)
    v = torch.empty(max(k, 1), dtype=a.dtype, device=dev)
    al = _dev_scalar(alpha, a.dtype, dev)
    be = _dev_scalar(beta, a.dtype, dev)
    call(f"b2s_csr_spgemm_numeric_{_SFX[a.dtype]}", n, m, _p(al), _p(a.row_ptrs),
         _p(a.col_idxs), _p(a.values), _p(b.row_ptrs), _p(b.col_idxs), _p(b.values), _p(be),
         _p(d.row_ptrs) if d is not None else None, _p(d.col_idxs) if d is not None else None,
         _p(d.values) if d is not None else None, _p(rp), _p(ci), _p(v), _p(ws), wsb, st)
    return Csr(a.exec, (n, m), rp, ci[:k], v[:k], a.strategy)


def spgeam(alpha, a: Csr, beta, b: Csr) -> Csr:
    """C = alpha A + beta B (csr::spgeam) for matrices with ascending
    columns: bit-exact with the reference executor."""
    if a.shape != b.shape:
        raise ValueError("A and B differ in shape (DimensionMismatch)")
    if a.dtype != b.dtype:
        raise TypeError("SpGEAM operands must share one value type")
    n = a.shape[0]
    dev = a.values.device
    wsb = lib().b2s_csr_spgeam_workspace_bytes(n)
    ws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)
    rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    nnz = C.c_int64(0)
    st = _stream(a.values)
    call("b2s_csr_spgeam_symbolic", n, _p(a.row_ptrs), _p(a.col_idxs), _p(b.row_ptrs),
         _p(b.col_idxs), _p(rp), C.byref(nnz), _p(ws), wsb, st)
    k = int(nnz.value)
    ci = torch.empty(max(k, 1), dtype=torch.int32, device=dev)
    v = torch.empty(max(k, 1), dtype=a.dtype, device=dev)
    al = _dev_scalar(alpha, a.dtype, dev)
    be = _dev_scalar(beta, a.dtype, dev)
    call(f"b2s_csr_spgeam_numeric_{_SFX[a.dtype]}", n, _p(al), _p(a.row_ptrs),
         _p(a.col_idxs), _p(a.values), _p(be), _p(b.row_ptrs), _p(b.col_idxs),
         _p(b.values), _p(rp), _p(ci), _p(v), st)
    return Csr(a.exec, a.shape, rp, ci[:k], v[:k], a.strategy)


class Hybrid(_SparseBase):
    """matrix::Hybrid (include/ginkgo/core/matrix/hybrid.hpp): an Ell part
    of `width` entries per row (column-major, stride >= rows, padding column
    -1) and a Coo part, sorted by row, with the rest of every longer row."""

    def __init__(self, exec_, shape, width, stride, ell_col_idxs, ell_values,
                 coo_row_idxs, coo_col_idxs, coo_values):
        self.exec = exec_
        self.shape = tuple(shape)
        self.width, self.stride = int(width), int(stride)
        self.ell_col_idxs, self.ell_values = ell_col_idxs, ell_values
        self.coo_row_idxs, self.coo_col_idxs = coo_row_idxs, coo_col_idxs
        self.coo_values = coo_values
        self.dtype = ell_values.dtype

    @property
    def coo_nnz(self):
        return int(self.coo_values.numel())

    def apply(self, *args):
        b2, x2, alpha, beta = self._apply_args(args)
        call(f"b2s_hybrid_spmv_{_SFX[self.dtype]}", self.shape[0], self.shape[1],
             self.width, self.stride, _p(self.ell_col_idxs), _p(self.ell_values),
             self.coo_nnz, _p(self.coo_row_idxs), _p(self.coo_col_idxs),
             _p(self.coo_values), _p(b2), b2.stride(0), _p(x2), x2.stride(0), x2.shape[1],
             _p(alpha), _p(beta), _stream(x2))
        return args[-1]

    def convert_to_csr(self) -> Csr:
        n = self.shape[0]
        dev = self.ell_values.device
        wsb = lib().b2s_hybrid_convert_workspace_bytes(n)
        ws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)
        rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
        nnz = C.c_int64(0)
        st = _stream(self.ell_values)
        call("b2s_hybrid_csr_row_ptrs", n, self.width, self.stride, _p(self.ell_col_idxs),
             self.coo_nnz, _p(self.coo_row_idxs), _p(rp), C.byref(nnz), _p(ws), wsb, st)
        k = int(nnz.value)
        ci = torch.empty(max(k, 1), dtype=torch.int32, device=dev)
        v = torch.empty(max(k, 1), dtype=self.dtype, device=dev)
        call(f"b2s_hybrid_convert_to_csr_{_SFX[self.dtype]}", n, self.width, self.stride,
             _p(self.ell_col_idxs), _p(self.ell_values), self.coo_nnz,
             _p(self.coo_row_idxs), _p(self.coo_col_idxs), _p(self.coo_values), _p(rp),
             _p(ci), _p(v), st)
        return Csr(self.exec, self.shape, rp, ci[:k], v[:k])


def _convert(t, dtype):
    """A contiguous copy of the 2-D block t in dtype, by the library."""
    out = torch.empty(t.shape, dtype=dtype, device=t.device)
    call("b2s_dense_convert", _VT[t.dtype], _VT[dtype], t.shape[0], t.shape[1],
         _p(t), t.stride(0), _p(out), out.stride(0), _stream(t))
    return out


_HYBRID = {"column_limit": 0, "imbalance_limit": 1, "imbalance_bounded_limit": 2,
           "minimal_storage_limit": 3, "automatic": 4}


def hybrid_config(row_nnz, strategy="automatic", num_columns=None, percent=None,
                  ratio=None, value_bytes=8, index_bytes=4):
    """(Ell width, Coo entries) of a Hybrid matrix with these row lengths
    under one of the reference's strategies (matrix::Hybrid::strategy_type,
    include/ginkgo/core/matrix/hybrid.hpp:103-360): column_limit(num_columns),
    imbalance_limit(percent=0.8), imbalance_bounded_limit(percent=0.8,
    ratio=0.0001), minimal_storage_limit(), automatic().  Host set-up in the
    library (b2s_hybrid_config)."""
    if strategy not in _HYBRID:
        raise ValueError(f"unknown Hybrid strategy {strategy!r}")
    p1 = {"column_limit": num_columns,
          "imbalance_limit": 0.8 if percent is None else percent,
          "imbalance_bounded_limit": 0.8 if percent is None else percent}.get(strategy, 0.0)
    p2 = 0.0001 if ratio is None else ratio
    if strategy == "column_limit" and num_columns is None:
        raise ValueError("column_limit needs num_columns")
    nnz = np.ascontiguousarray(row_nnz, dtype=np.int64)
    buf = nnz if len(nnz) else np.zeros(1, dtype=np.int64)
    out = np.zeros(2, dtype=np.int64)
    call("b2s_hybrid_config", len(nnz), buf.ctypes.data, _HYBRID[strategy], float(p1),
         float(p2), int(value_bytes), int(index_bytes), out.ctypes.data)
    return int(out[0]), int(out[1])
