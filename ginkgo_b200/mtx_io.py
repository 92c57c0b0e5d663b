"""MatrixMarket and binary matrix I/O, named after the reference's
``gko::read_raw`` / ``write_raw`` / ``read_binary_raw`` / ``write_binary_raw``
/ ``read_generic_raw`` (include/ginkgo/core/base/mtx_io.hpp) and
``gko::read<MatrixType>`` / ``gko::write`` for a Csr.

The parsing and formatting run in the C++ library (``b2s_mtx_*``, host code);
this module moves bytes and numpy arrays across the C ABI.  Matrix data is a
``MatrixData``: ``size`` (rows, cols) and parallel arrays ``row_idxs``,
``col_idxs``, ``values`` (0-based, the reference's matrix_data nonzeros).
Reading raises ``GinkgoError`` with the reference's StreamError message on
malformed input.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from ._lib import call

_VT = {np.dtype(np.float64): 0, np.dtype(np.float32): 1}
_IT = {np.dtype(np.int32): 0, np.dtype(np.int64): 1}
TEXT, BINARY, GENERIC, COORDINATE, ARRAY = 0, 1, 2, 3, 4


@dataclass
class MatrixData:
    """gko::matrix_data: size and (row, column, value) entries."""
    size: tuple
    row_idxs: np.ndarray
    col_idxs: np.ndarray
    values: np.ndarray

    @property
    def nonzeros(self):
        """The entries as (row, column, value) tuples."""
        return list(zip(self.row_idxs.tolist(), self.col_idxs.tolist(),
                        self.values.tolist()))

    @staticmethod
    def from_entries(size, entries, value_type=np.float64, index_type=np.int32):
        """Matrix data with the given (row, column, value) entries, in order."""
        e = list(entries)
        return MatrixData((int(size[0]), int(size[1])),
                          np.array([t[0] for t in e], dtype=index_type),
                          np.array([t[1] for t in e], dtype=index_type),
                          np.array([t[2] for t in e], dtype=value_type))


def _bytes(src):
    if isinstance(src, (bytes, bytearray, memoryview)):
        return bytes(src)
    if isinstance(src, str):
        return src.encode()
    if isinstance(src, os.PathLike):
        with open(src, "rb") as f:
            return f.read()
    if hasattr(src, "read"):
        data = src.read()
        return data.encode() if isinstance(data, str) else bytes(data)
    raise TypeError("expected bytes, str, a path or a readable object")


def _take(handle, value_type, index_type):
    try:
        sizes = np.zeros(4, dtype=np.int64)
        call("b2s_mtx_sizes", handle, sizes.ctypes.data)
        n = int(sizes[2])
        r = np.empty(n, dtype=index_type)
        c = np.empty(n, dtype=index_type)
        v = np.empty(n, dtype=value_type)
        out = np.empty(int(sizes[3]), dtype=np.uint8)
        call("b2s_mtx_copy", handle, r.ctypes.data, c.ctypes.data, v.ctypes.data,
             out.ctypes.data)
        return (int(sizes[0]), int(sizes[1])), r, c, v, out.tobytes()
    finally:
        call("b2s_mtx_free", handle)


def _read(src, fmt, value_type, index_type):
    vt, it = np.dtype(value_type), np.dtype(index_type)
    if vt not in _VT or it not in _IT:
        raise TypeError("value type float64/float32 and index type int32/int64 only")
    data = _bytes(src)  # ctypes hands a bytes object's own buffer to void*
    h = C.c_void_p()
    call("b2s_mtx_read", data, len(data), fmt, _VT[vt], _IT[it], C.addressof(h))
    size, r, c, v, _ = _take(h, vt, it)
    return MatrixData(size, r, c, v)


def read_raw(src, value_type=np.float64, index_type=np.int32) -> MatrixData:
    """MatrixMarket text (core/base/mtx_io.cpp:747-751): entries sorted by
    (row, column), symmetric storage expanded."""
    return _read(src, TEXT, value_type, index_type)


def read_binary_raw(src, value_type=np.float64, index_type=np.int32) -> MatrixData:
    """The reference's binary format (core/base/mtx_io.cpp:882-927)."""
    return _read(src, BINARY, value_type, index_type)


def read_generic_raw(src, value_type=np.float64, index_type=np.int32) -> MatrixData:
    """Text when the input starts with '%', else binary (mtx_io.cpp:930-941)."""
    return _read(src, GENERIC, value_type, index_type)


def _write(data: MatrixData, fmt) -> bytes:
    vt, it = data.values.dtype, data.row_idxs.dtype
    if vt not in _VT or it not in _IT or data.col_idxs.dtype != it:
        raise TypeError("value type float64/float32 and index type int32/int64 only")
    r = np.ascontiguousarray(data.row_idxs)
    c = np.ascontiguousarray(data.col_idxs)
    v = np.ascontiguousarray(data.values)
    if not (len(r) == len(c) == len(v)):
        raise ValueError("row, column and value arrays differ in length")
    h = C.c_void_p()
    call("b2s_mtx_write", int(data.size[0]), int(data.size[1]), len(r), r.ctypes.data,
         c.ctypes.data, v.ctypes.data, _VT[vt], _IT[it], fmt, C.addressof(h))
    return _take(h, vt, it)[4]


def write_raw(data: MatrixData, layout: str = "coordinate") -> str:
    """MatrixMarket text, 'coordinate' or 'array' layout, real general
    (core/base/mtx_io.cpp:980-1004)."""
    if layout not in ("coordinate", "array"):
        raise ValueError("layout is 'coordinate' or 'array'")
    return _write(data, ARRAY if layout == "array" else COORDINATE).decode()


def write_binary_raw(data: MatrixData) -> bytes:
    """The reference's binary format (core/base/mtx_io.cpp:943-978)."""
    return _write(data, BINARY)


def data_to_csr_arrays(data: MatrixData):
    """Csr arrays (row_ptrs, col_idxs, values; int32 indices) of matrix data
    sorted by row, as Csr::read does with matrix_data (entries with equal
    coordinates are kept, so the SpMV adds them).  Every index must lie inside
    the size."""
    n, m = data.size
    r = np.asarray(data.row_idxs, dtype=np.int64)
    c = np.asarray(data.col_idxs, dtype=np.int64)
    if n >= 2**31 or m >= 2**31 or len(r) >= 2**31:
        raise ValueError("Csr with int32 indices holds < 2^31 rows, columns and entries")
    if len(r) and (r.min() < 0 or r.max() >= n or c.min() < 0 or c.max() >= m):
        raise ValueError("matrix data has an entry outside its size")
    if len(r) > 1 and np.any(np.diff(r) < 0):
        raise ValueError("matrix data is not sorted by row")
    rp = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return rp, c.astype(np.int32), np.asarray(data.values)


def read(matrix_type, src, exec_, dtype=None, **convert_args):
    """gko::read<MatrixType>(stream, exec) for Csr, Ell or Sellp: MatrixMarket
    text or the binary format (read_generic_raw), then Csr::read; Ell and
    Sellp are converted from the Csr on the device (convert_args go to
    convert_to_sellp: slice_size, stride_factor)."""
    import torch
    from .matrix import Csr, Ell, Sellp
    if matrix_type not in (Csr, Ell, Sellp):
        raise TypeError("read() builds a Csr, Ell or Sellp")
    dtype = torch.float64 if dtype is None else dtype
    vt = np.float64 if dtype == torch.float64 else np.float32
    data = read_generic_raw(src, vt, np.int32)
    rp, ci, v = data_to_csr_arrays(data)
    A = Csr.read(exec_, rp, ci, v, shape=data.size, dtype=dtype)
    if matrix_type is Ell:
        return A.convert_to_ell()
    if matrix_type is Sellp:
        return A.convert_to_sellp(**convert_args)
    return A


def write(csr, layout: str | None = None) -> str:
    """gko::write(stream, matrix) for a Csr: array layout when at least a
    quarter of the entries are stored, else coordinate (mtx_io.cpp:1043-1047)."""
    rp = csr.row_ptrs.cpu().numpy().astype(np.int64)
    n, m = csr.shape
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    data = MatrixData((n, m), rows, csr.col_idxs.cpu().numpy().astype(np.int32),
                      csr.values.cpu().numpy())
    if layout is None:
        layout = "array" if len(rows) >= n * m // 4 else "coordinate"
    return write_raw(data, layout)


def read_dense(src, exec_=None, dtype=None):
    """gko::read<Dense>(stream, exec): the file as a dense rows x cols torch
    tensor (row-major, the layout of the right-hand sides and solutions on
    this path), zero where the file has no entry; an entry given twice keeps
    the later one (Dense::read, core/matrix/dense.cpp:1064-1072).  On
    exec_'s device when one is given, else on the host."""
    import torch
    dtype = torch.float64 if dtype is None else dtype
    vt = np.float64 if dtype == torch.float64 else np.float32
    data = read_generic_raw(src, vt, np.int64)
    n, m = data.size
    r, c = data.row_idxs, data.col_idxs
    if len(r) and (r.min() < 0 or r.max() >= n or c.min() < 0 or c.max() >= m):
        raise ValueError("matrix data has an entry outside its size")
    out = np.zeros((n, m), dtype=vt)
    # the entries come sorted by (row, column) with a repeated position in
    # file order, so the last of each run is the later value
    last = np.ones(len(r), dtype=bool)
    last[:-1] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    out[r[last], c[last]] = data.values[last]
    t = torch.from_numpy(out)
    return t.to(exec_.device) if exec_ is not None else t


def write_dense(tensor, layout: str | None = None) -> str:
    """gko::write(stream, Dense): the nonzero entries in row-major order
    (Dense::write, core/matrix/dense.cpp:1119-1132), array layout when at
    least a quarter of the entries are nonzero, else coordinate
    (mtx_io.cpp:1043-1047).  A 1-D tensor is one column."""
    a = tensor.detach().cpu().numpy()
    if a.ndim == 1:
        a = a[:, None]
    if a.dtype not in (np.float64, np.float32):
        a = a.astype(np.float64)
    n, m = a.shape
    r, c = np.nonzero(a)  # NaN counts as nonzero, as is_nonzero does
    data = MatrixData((n, m), r.astype(np.int64), c.astype(np.int64), a[r, c])
    if layout is None:
        layout = "array" if len(r) >= n * m // 4 else "coordinate"
    return write_raw(data, layout)
