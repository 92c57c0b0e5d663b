"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (built by oracle/Makefile) and exposes numpy
wrappers.  Only tests, the smoke check and the benchmark's CPU-baseline leg
import this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_p = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int
_f64 = C.c_double


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        for s in ("f64", "f32"):
            getattr(_lib, f"orc_csr_spmv_{s}").argtypes = [
                _i64, _p, _p, _p, _p, _i64, _p, _i64, _i64, _p, _p]
            getattr(_lib, f"orc_csr_spmv_par_{s}").argtypes = [
                _i64, _p, _p, _p, _p, _i64, _p, _i64, _i64, _i32]
            getattr(_lib, f"orc_ell_spmv_{s}").argtypes = [
                _i64, _i64, _i64, _p, _p, _p, _i64, _p, _i64, _i64, _p, _p]
            getattr(_lib, f"orc_sellp_spmv_{s}").argtypes = [
                _i64, _i64, _p, _p, _p, _p, _p, _i64, _p, _i64, _i64, _p, _p]
            getattr(_lib, f"orc_csr_to_ell_{s}").argtypes = [
                _i64, _p, _p, _p, _i64, _i64, _p, _p]
            getattr(_lib, f"orc_csr_to_sellp_{s}").argtypes = [
                _i64, _p, _p, _p, _i64, _p, _p, _p, _p]
            getattr(_lib, f"orc_csr_transpose_{s}").argtypes = [
                _i64, _i64, _p, _p, _p, _p, _p, _p]
            getattr(_lib, f"orc_jacobi_invert_diagonal_{s}").argtypes = [
                _i64, _p, _p, _p, _p]
            getattr(_lib, f"orc_cg_step_1_{s}").argtypes = [
                _i64, _i64, _p, _p, _p, _p, _p]
            getattr(_lib, f"orc_cg_step_2_{s}").argtypes = [
                _i64, _i64, _p, _p, _p, _p, _p, _p, _p]
            getattr(_lib, f"orc_gmres_hessenberg_qr_{s}").argtypes = [
                _i64, _i64, _p, _p, _p, _p, _p, _p, _p]
            getattr(_lib, f"orc_gmres_solve_krylov_{s}").argtypes = [
                _i64, _p, _p, _i64, _p, _p, _p]
            f = getattr(_lib, f"orc_cg_{s}")
            f.argtypes = [_i64, _p, _p, _p, _p, _p, _p, _i64, _i32, _f64, _i32, _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_cg_block_{s}")
            f.argtypes = [_i64, _p, _p, _p, _i64, _p, _i32, _p, _p, _p, _i64, _i32, _f64,
                          _i32, _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_bicgstab_{s}")
            f.argtypes = [_i64, _p, _p, _p, _p, _p, _p, _i32, _f64, _i32, _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_bicgstab_block_{s}")
            f.argtypes = [_i64, _p, _p, _p, _i64, _p, _i32, _p, _p, _p, _i32, _f64, _i32,
                          _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_gmres_{s}")
            f.argtypes = [_i64, _p, _p, _p, _p, _p, _p, _i32, _i32, _i32, _f64, _i32,
                          _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_gmres_block_{s}")
            f.argtypes = [_i64, _p, _p, _p, _i64, _p, _i32, _p, _p, _p, _i32, _i32, _i32,
                          _f64, _i32, _p, _p]
            f.restype = _i32
            f = getattr(_lib, f"orc_batch_bicgstab_ell_{s}")
            f.argtypes = [_i64, _i64, _i64, _p, _p, _p, _p, _i32, _f64, _i32,
                          _p, _p]
            f.restype = _i32
        _lib.orc_sellp_compute_slice_sets.argtypes = [_i64, _p, _i64, _i64, _p, _p]
        _lib.orc_csr_max_row_nnz.argtypes = [_i64, _p]
        _lib.orc_csr_max_row_nnz.restype = _i64
        _lib.orc_ir_gmres_mixed.argtypes = [
            _i64, _p, _p, _p, _p, _p, _i32, _i32, _f64, _i32, _f64, _p, _p, _p]
        _lib.orc_ir_gmres_mixed.restype = _i32
    return _lib


def _ptr(a):
    # data_as keeps a reference to the array alive inside the pointer object
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _sfx(dtype):
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[np.dtype(dtype)]


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _as2d(x):
    return x.reshape(x.shape[0], -1)


def csr_spmv(rp, ci, v, x, y=None, alpha=None, beta=None):
    """y = A x, or y = alpha A x + beta y when alpha/beta are given."""
    v = np.ascontiguousarray(v)
    dt = v.dtype
    rp, ci = _c(rp, np.int32), _c(ci, np.int32)
    x2 = _as2d(_c(x, dt))
    n, k = len(rp) - 1, x2.shape[1]
    y2 = np.zeros((n, k), dt) if y is None else _as2d(_c(y, dt)).copy()
    a = None if alpha is None else np.array([alpha], dt)
    b = None if beta is None else np.array([beta], dt)
    getattr(lib(), f"orc_csr_spmv_{_sfx(dt)}")(
        n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x2), k, _ptr(y2), k, k, _ptr(a), _ptr(b))
    return y2.reshape((n,) + tuple(np.shape(x)[1:]))


def csr_spmv_par(rp, ci, v, x, y, nthreads):
    """Threaded y = A x in place (the timed CPU baseline)."""
    k = 1 if x.ndim == 1 else x.shape[1]
    getattr(lib(), f"orc_csr_spmv_par_{_sfx(v.dtype)}")(
        len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), k, _ptr(y), k, k,
        int(nthreads))


def ell_spmv(n, width, stride, ci, v, x, y=None, alpha=None, beta=None):
    v = np.ascontiguousarray(v)
    dt = v.dtype
    x2 = _as2d(_c(x, dt))
    k = x2.shape[1]
    y2 = np.zeros((n, k), dt) if y is None else _as2d(_c(y, dt)).copy()
    a = None if alpha is None else np.array([alpha], dt)
    b = None if beta is None else np.array([beta], dt)
    getattr(lib(), f"orc_ell_spmv_{_sfx(dt)}")(
        n, width, stride, _ptr(_c(ci, np.int32)), _ptr(v), _ptr(x2), k, _ptr(y2),
        k, k, _ptr(a), _ptr(b))
    return y2.reshape((n,) + tuple(np.shape(x)[1:]))


def sellp_spmv(n, slice_size, slice_sets, slice_lengths, ci, v, x, y=None,
               alpha=None, beta=None):
    v = np.ascontiguousarray(v)
    dt = v.dtype
    x2 = _as2d(_c(x, dt))
    k = x2.shape[1]
    y2 = np.zeros((n, k), dt) if y is None else _as2d(_c(y, dt)).copy()
    a = None if alpha is None else np.array([alpha], dt)
    b = None if beta is None else np.array([beta], dt)
    getattr(lib(), f"orc_sellp_spmv_{_sfx(dt)}")(
        n, slice_size, _ptr(_c(slice_sets, np.uint64)),
        _ptr(_c(slice_lengths, np.uint64)), _ptr(_c(ci, np.int32)), _ptr(v),
        _ptr(x2), k, _ptr(y2), k, k, _ptr(a), _ptr(b))
    return y2.reshape((n,) + tuple(np.shape(x)[1:]))


def max_row_nnz(rp):
    rp = _c(rp, np.int32)
    return int(lib().orc_csr_max_row_nnz(len(rp) - 1, _ptr(rp)))


def csr_to_ell(rp, ci, v, width=None, stride=None):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    n = len(rp) - 1
    width = max_row_nnz(rp) if width is None else width
    stride = n if stride is None else stride
    eci = np.empty(width * stride, np.int32)
    ev = np.empty(width * stride, v.dtype)
    getattr(lib(), f"orc_csr_to_ell_{_sfx(v.dtype)}")(
        n, _ptr(rp), _ptr(ci), _ptr(v), width, stride, _ptr(eci), _ptr(ev))
    return width, stride, eci, ev


def sellp_slice_sets(rp, slice_size=64, stride_factor=1):
    rp = _c(rp, np.int32)
    n = len(rp) - 1
    ns = (n + slice_size - 1) // slice_size
    sets = np.zeros(ns + 1, np.uint64)
    lens = np.zeros(ns, np.uint64)
    lib().orc_sellp_compute_slice_sets(n, _ptr(rp), slice_size, stride_factor,
                                       _ptr(sets), _ptr(lens))
    return sets, lens


def csr_to_sellp(rp, ci, v, slice_size=64, stride_factor=1):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    n = len(rp) - 1
    sets, lens = sellp_slice_sets(rp, slice_size, stride_factor)
    total = int(sets[-1]) * slice_size
    sci = np.full(total, -1, np.int32)
    sv = np.zeros(total, v.dtype)
    getattr(lib(), f"orc_csr_to_sellp_{_sfx(v.dtype)}")(
        n, _ptr(rp), _ptr(ci), _ptr(v), slice_size, _ptr(sets), _ptr(lens),
        _ptr(sci), _ptr(sv))
    return sets, lens, sci, sv


def csr_transpose(rp, ci, v, ncols):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    nnz = int(rp[-1])
    trp = np.empty(ncols + 1, np.int32)
    tci = np.empty(nnz, np.int32)
    tv = np.empty(nnz, v.dtype)
    getattr(lib(), f"orc_csr_transpose_{_sfx(v.dtype)}")(
        len(rp) - 1, ncols, _ptr(rp), _ptr(ci), _ptr(v), _ptr(trp), _ptr(tci),
        _ptr(tv))
    return trp, tci, tv


def jacobi_invert_diagonal(rp, ci, v):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    out = np.empty(len(rp) - 1, v.dtype)
    getattr(lib(), f"orc_jacobi_invert_diagonal_{_sfx(v.dtype)}")(
        len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), _ptr(out))
    return out


# residual criterion modes: baseline (0 rhs_norm, 1 initial_resnorm,
# 2 absolute) plus 4 for the implicit residual norm
MODES = {"rhs_norm": 0, "initial_resnorm": 1, "absolute": 2}
IMPLICIT = 4
ORTHO = {"mgs": 0, "cgs": 1, "cgs2": 2}


def cg(rp, ci, v, b, x0=None, jacobi=True, max_iters=1000, reduction=1e-10, mode=0):
    """Returns (x, iterations, residual norms, converged columns)."""
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b2 = _as2d(_c(b, dt))
    n, k = b2.shape
    x = np.zeros((n, k), dt) if x0 is None else _as2d(_c(x0, dt)).copy()
    inv = jacobi_invert_diagonal(rp, ci, v) if jacobi else None
    it = C.c_int(0)
    res = np.zeros(k, np.float64)
    conv = getattr(lib(), f"orc_cg_{_sfx(dt)}")(
        n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(inv), _ptr(b2), _ptr(x), k,
        max_iters, reduction, int(mode), C.byref(it), _ptr(res))
    return x.reshape(np.shape(b)), it.value, res, conv


def _block_inverses(block_ptrs, blocks, max_block_size, dt):
    """The inverses as one [num_blocks, m, m] array (block i in the top-left
    corner of slot i), the layout of the oracle's block preconditioners."""
    m = int(max_block_size)
    ptrs = _c(block_ptrs, np.int32)
    binv = np.zeros((len(ptrs) - 1, m, m), dt)
    for i, blk in enumerate(blocks):
        s = np.asarray(blk).shape[0]
        binv[i, :s, :s] = blk
    return ptrs, binv


def bicgstab_block(rp, ci, v, b, block_ptrs, blocks, max_block_size, x0=None,
                   max_iters=1000, reduction=1e-10, mode=0):
    """BiCGStab (one right-hand side) with a block Jacobi preconditioner;
    block arguments as cg_block, returns as bicgstab."""
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b = _c(b, dt)
    x = np.zeros_like(b) if x0 is None else _c(x0, dt).copy()
    ptrs, binv = _block_inverses(block_ptrs, blocks, max_block_size, dt)
    it = C.c_int(0)
    res = C.c_double(0)
    conv = getattr(lib(), f"orc_bicgstab_block_{_sfx(dt)}")(
        len(b), _ptr(rp), _ptr(ci), _ptr(v), len(ptrs) - 1, _ptr(ptrs), int(max_block_size),
        _ptr(binv), _ptr(b), _ptr(x), max_iters, reduction, int(mode), C.byref(it),
        C.byref(res))
    return x, it.value, res.value, conv


def cg_block(rp, ci, v, b, block_ptrs, blocks, max_block_size, x0=None, max_iters=1000,
             reduction=1e-10, mode=0):
    """CG with a block Jacobi preconditioner: block_ptrs delimit the blocks,
    blocks[i] is block i's inverse (square, its block's size), as
    oracle.jacobi.generate returns them.  Returns as cg."""
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b2 = _as2d(_c(b, dt))
    n, k = b2.shape
    x = np.zeros((n, k), dt) if x0 is None else _as2d(_c(x0, dt)).copy()
    m = int(max_block_size)
    ptrs, binv = _block_inverses(block_ptrs, blocks, m, dt)
    it = C.c_int(0)
    res = np.zeros(k, np.float64)
    conv = getattr(lib(), f"orc_cg_block_{_sfx(dt)}")(
        n, _ptr(rp), _ptr(ci), _ptr(v), len(ptrs) - 1, _ptr(ptrs), m, _ptr(binv), _ptr(b2),
        _ptr(x), k, max_iters, reduction, int(mode), C.byref(it), _ptr(res))
    return x.reshape(np.shape(b)), it.value, res, conv


def bicgstab(rp, ci, v, b, x0=None, jacobi=True, max_iters=1000, reduction=1e-10,
             mode=0):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b = _c(b, dt)
    x = np.zeros_like(b) if x0 is None else _c(x0, dt).copy()
    inv = jacobi_invert_diagonal(rp, ci, v) if jacobi else None
    it = C.c_int(0)
    res = C.c_double(0)
    conv = getattr(lib(), f"orc_bicgstab_{_sfx(dt)}")(
        len(b), _ptr(rp), _ptr(ci), _ptr(v), _ptr(inv), _ptr(b), _ptr(x),
        max_iters, reduction, int(mode), C.byref(it), C.byref(res))
    return x, it.value, res.value, conv


def gmres(rp, ci, v, b, x0=None, jacobi=True, krylov_dim=30, max_iters=1000,
          reduction=1e-10, ortho="mgs", mode=0):
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b = _c(b, dt)
    x = np.zeros_like(b) if x0 is None else _c(x0, dt).copy()
    inv = jacobi_invert_diagonal(rp, ci, v) if jacobi else None
    it = C.c_int(0)
    res = C.c_double(0)
    conv = getattr(lib(), f"orc_gmres_{_sfx(dt)}")(
        len(b), _ptr(rp), _ptr(ci), _ptr(v), _ptr(inv), _ptr(b), _ptr(x),
        krylov_dim, ORTHO[ortho], max_iters, reduction, int(mode), C.byref(it),
        C.byref(res))
    return x, it.value, res.value, conv


def gmres_block(rp, ci, v, b, block_ptrs, blocks, max_block_size, x0=None, krylov_dim=30,
                max_iters=1000, reduction=1e-10, ortho="mgs", mode=0):
    """GMRES with a block Jacobi preconditioner; block arguments as
    cg_block, returns as gmres."""
    rp, ci, v = _c(rp, np.int32), _c(ci, np.int32), np.ascontiguousarray(v)
    dt = v.dtype
    b = _c(b, dt)
    x = np.zeros_like(b) if x0 is None else _c(x0, dt).copy()
    ptrs, binv = _block_inverses(block_ptrs, blocks, max_block_size, dt)
    it = C.c_int(0)
    res = C.c_double(0)
    conv = getattr(lib(), f"orc_gmres_block_{_sfx(dt)}")(
        len(b), _ptr(rp), _ptr(ci), _ptr(v), len(ptrs) - 1, _ptr(ptrs), int(max_block_size),
        _ptr(binv), _ptr(b), _ptr(x), krylov_dim, ORTHO[ortho], max_iters, reduction,
        int(mode), C.byref(it), C.byref(res))
    return x, it.value, res.value, conv


def ir_gmres_mixed(rp, ci, v, b, krylov_dim=30, inner_iters=30,
                   inner_reduction=1e-4, max_outer=100, reduction=1e-10):
    rp, ci = _c(rp, np.int32), _c(ci, np.int32)
    v, b = _c(v, np.float64), _c(b, np.float64)
    x = np.zeros_like(b)
    outer, inner = C.c_int(0), C.c_int(0)
    res = C.c_double(0)
    conv = lib().orc_ir_gmres_mixed(
        len(b), _ptr(rp), _ptr(ci), _ptr(v), _ptr(b), _ptr(x), krylov_dim,
        inner_iters, inner_reduction, max_outer, reduction, C.byref(outer),
        C.byref(inner), C.byref(res))
    return x, outer.value, inner.value, res.value, conv


def batch_bicgstab_ell(n, width, stride, ci, v, b, x0=None, max_iters=500,
                       tol=1e-8, jacobi=True):
    v = np.ascontiguousarray(v)
    dt = v.dtype
    b = _c(b, dt)
    x = np.zeros_like(b) if x0 is None else _c(x0, dt).copy()
    it = C.c_int(0)
    res = C.c_double(0)
    conv = getattr(lib(), f"orc_batch_bicgstab_ell_{_sfx(dt)}")(
        n, width, stride, _ptr(_c(ci, np.int32)), _ptr(v), _ptr(b), _ptr(x),
        max_iters, tol, int(jacobi), C.byref(it), C.byref(res))
    return x, it.value, res.value, conv


def cg_step_1(p, z, rho, prev_rho, stopped):
    """In-place CG step 1 on row-major (n, k) arrays."""
    dt = p.dtype
    n, k = p.shape
    st = np.ascontiguousarray(stopped, np.int8)
    getattr(lib(), f"orc_cg_step_1_{_sfx(dt)}")(
        n, k, _ptr(p), _ptr(_c(z, dt)), _ptr(_c(rho, dt)), _ptr(_c(prev_rho, dt)),
        _ptr(st))


def cg_step_2(x, r, p, q, beta, rho, stopped):
    dt = x.dtype
    n, k = x.shape
    st = np.ascontiguousarray(stopped, np.int8)
    getattr(lib(), f"orc_cg_step_2_{_sfx(dt)}")(
        n, k, _ptr(x), _ptr(r), _ptr(_c(p, dt)), _ptr(_c(q, dt)),
        _ptr(_c(beta, dt)), _ptr(_c(rho, dt)), _ptr(st))


def gmres_hessenberg_qr(iteration, givens_sin, givens_cos, residual_norm, rnc,
                        hessenberg_iter, final_iter_nums, stopped):
    """In-place Givens update (arrays row-major, k = number of columns)."""
    dt = givens_sin.dtype
    k = givens_sin.shape[1]
    st = np.ascontiguousarray(stopped, np.int8)
    getattr(lib(), f"orc_gmres_hessenberg_qr_{_sfx(dt)}")(
        k, iteration, _ptr(givens_sin), _ptr(givens_cos), _ptr(residual_norm),
        _ptr(rnc), _ptr(hessenberg_iter), _ptr(final_iter_nums), _ptr(st))


def gmres_solve_krylov(rnc, hessenberg, final_iter_nums):
    dt = hessenberg.dtype
    k = rnc.shape[1]
    y = np.zeros((int(np.max(final_iter_nums)), k), dt)
    getattr(lib(), f"orc_gmres_solve_krylov_{_sfx(dt)}")(
        k, _ptr(_c(rnc, dt)), _ptr(_c(hessenberg, dt)), hessenberg.shape[1],
        _ptr(y), _ptr(np.ascontiguousarray(final_iter_nums, np.int64)), None)
    return y
