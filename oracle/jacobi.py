"""Pure-Python restatement of the reference's block Jacobi preconditioner
(core/preconditioner/jacobi.cpp with reference/preconditioner/
jacobi_kernels.cpp) — TEST INFRASTRUCTURE ONLY.

The checker for a future device block Jacobi: block detection (natural
blocks of rows with equal patterns, then supervariable agglomeration under
max_block_size), extraction and in-place Gauss-Jordan inversion with partial
pivoting of each diagonal block, its application (plain and alpha D^-1 b +
beta x), transposition, conversion to dense, scalar Jacobi, and the L1
modifications.  Full-precision block storage only (no adaptive precision).
Pinned by the reference's own tests (reference/test/preconditioner/
jacobi_kernels.cpp).  Only tests import this module.

Matrices are Csr arrays (row_ptrs, col_idxs, values), sorted by column in
each row.  Inverted blocks are dense row-major numpy arrays.
"""
from __future__ import annotations

import numpy as np


def find_blocks(rp, ci, max_block_size):
    """find_natural_blocks + agglomerate_supervariables (jacobi_kernels.cpp:
    28-98): block pointers."""
    n = len(rp) - 1
    if n == 0:
        return [0]
    ptrs = [0]
    size = 1
    for i in range(1, n):
        prev = list(ci[rp[i - 1]:rp[i]])
        cur = list(ci[rp[i]:rp[i + 1]])
        if size < max_block_size and prev == cur:
            size += 1
        else:
            ptrs.append(ptrs[-1] + size)
            size = 1
    ptrs.append(ptrs[-1] + size)
    # agglomerate neighbouring natural blocks up to max_block_size
    out = [0]
    cur = ptrs[1] - ptrs[0]
    for i in range(1, len(ptrs) - 1):
        bs = ptrs[i + 1] - ptrs[i]
        if cur + bs <= max_block_size:
            cur += bs
        else:
            out.append(ptrs[i])
            cur = bs
    out.append(ptrs[-1])
    return out


def extract_block(rp, ci, v, start, size, dtype=np.float64):
    """extract_block (:100-125): the dense diagonal block."""
    blk = np.zeros((size, size), dtype=dtype)
    for r in range(size):
        for k in range(rp[start + r], rp[start + r + 1]):
            c = ci[k] - start
            if 0 <= c < size:
                blk[r, c] = v[k]
    return blk


def invert_block(blk):
    """invert_block (:223-240) with choose_pivot, swap_rows and
    apply_gauss_jordan_transform (:128-170), then permute_and_transpose_block
    (:203-220): in-place Gauss-Jordan with partial pivoting.  Returns the
    inverse (row-major).  A zero pivot ends the elimination and the block is
    stored as far as it got, as the reference's generate does (it does not
    check invert_block's result)."""
    b = np.array(blk, copy=True)
    dt = b.dtype.type
    n = b.shape[0]
    perm = list(range(n))
    for k in range(n):
        cp = k
        for i in range(k + 1, n):  # first strictly larger magnitude wins
            if abs(b[cp, k]) < abs(b[i, k]):
                cp = i
        b[[k, cp]] = b[[cp, k]]
        perm[k], perm[cp] = perm[cp], perm[k]
        d = b[k, k]
        if d == 0:
            break
        for i in range(n):
            b[i, k] = dt(b[i, k] / -d)
        b[k, k] = 0
        for i in range(n):
            for j in range(n):
                b[i, j] = dt(b[i, j] + b[i, k] * b[k, j])
        for j in range(n):
            b[k, j] = dt(b[k, j] / d)
        b[k, k] = dt(1 / d)
    inv = np.zeros_like(b)
    for i in range(n):
        for j in range(n):
            inv[i, perm[j]] = b[i, j]
    return inv


def scalar_l1(rp, ci, v, diag):
    """scalar_l1 (:727-745): diag[row] += sum of |off-diagonal| entries."""
    out = np.array(diag, copy=True)
    for r in range(len(rp) - 1):
        out[r] += sum(abs(v[k]) for k in range(rp[r], rp[r + 1]) if ci[k] != r)
    return out


def block_l1(rp, ci, v, block_ptrs):
    """block_l1 (:751-779): each row's diagonal entry gains the absolute sum
    of its entries outside the row's block (the diagonal must be stored).
    Returns the new values."""
    out = np.array(v, copy=True)
    for s, e in zip(block_ptrs[:-1], block_ptrs[1:]):
        for r in range(s, e):
            off, d = 0.0, -1
            for k in range(rp[r], rp[r + 1]):
                if s <= ci[k] < e:
                    if ci[k] == r:
                        d = k
                    continue
                off += abs(v[k])
            out[d] += off
    return out


def _with_diagonal(rp, ci, v):
    """add_diagonal_elements: every row gets a (zero) diagonal entry where
    none is stored, columns kept sorted."""
    n = len(rp) - 1
    nrp, nci, nv = [0], [], []
    for r in range(n):
        cols = list(ci[rp[r]:rp[r + 1]])
        vals = list(v[rp[r]:rp[r + 1]])
        if r not in cols:
            pos = int(np.searchsorted(cols, r))
            cols.insert(pos, r)
            vals.insert(pos, 0.0)
        nci += cols
        nv += vals
        nrp.append(len(nci))
    return np.array(nrp), np.array(nci), np.array(nv)


def generate(rp, ci, v, max_block_size=32, block_ptrs=None, aggregate_l1=False,
             dtype=np.float64):
    """Jacobi::generate (core/preconditioner/jacobi.cpp:336-420): returns
    ("scalar", inverse diagonal) for max_block_size 1 (a zero diagonal
    entry inverts to 1, jacobi_kernels invert_diagonal), else ("block",
    block_ptrs, [inverse blocks])."""
    n = len(rp) - 1
    v = np.asarray(v, dtype=dtype)
    if max_block_size == 1:
        diag = np.zeros(n, dtype=dtype)
        for r in range(n):
            for k in range(rp[r], rp[r + 1]):
                if ci[k] == r:
                    diag[r] = v[k]
        if aggregate_l1:
            diag = scalar_l1(rp, ci, v, diag)
        inv = np.array([dtype(1) if d == 0 else dtype(1) / d for d in diag], dtype=dtype)
        return "scalar", inv
    ptrs = list(block_ptrs) if block_ptrs is not None else find_blocks(rp, ci, max_block_size)
    if aggregate_l1:
        rp, ci, v = _with_diagonal(rp, ci, v)
        v = block_l1(rp, ci, v, ptrs).astype(dtype)
    blocks = [invert_block(extract_block(rp, ci, v, s, e - s, dtype))
              for s, e in zip(ptrs[:-1], ptrs[1:])]
    return "block", ptrs, blocks


def apply(prec, b, x=None, alpha=None, beta=None):
    """apply / simple_apply (:395-470, apply_block) and the scalar forms:
    x = D^-1 b, or x = alpha D^-1 b + beta x (beta = 0 ignores x)."""
    b = np.asarray(b)
    one = b.ndim == 1
    b2 = b.reshape(len(b), -1)
    dt = b2.dtype.type
    out = np.zeros_like(b2) if x is None else np.array(x, dtype=b2.dtype).reshape(b2.shape)
    a = dt(1) if alpha is None else dt(alpha)
    be = dt(0) if beta is None else dt(beta)
    if prec[0] == "scalar":
        inv = prec[1]
        for r in range(b2.shape[0]):
            for c in range(b2.shape[1]):
                out[r, c] = (be * out[r, c] if x is not None else 0) + a * b2[r, c] * inv[r]
    else:
        _, ptrs, blocks = prec
        for (s, e), inv in zip(zip(ptrs[:-1], ptrs[1:]), blocks):
            seg = out[s:e] * be if be != 0 else np.zeros_like(out[s:e])
            for inner in range(e - s):
                for row in range(e - s):
                    seg[row] = seg[row] + a * inv[row, inner] * b2[s + inner]
            out[s:e] = seg
    return out[:, 0] if one else out


def transpose(prec):
    """Jacobi::transpose: every inverse block transposed."""
    if prec[0] == "scalar":
        return prec
    _, ptrs, blocks = prec
    return "block", ptrs, [blk.T.copy() for blk in blocks]


def to_dense(prec, n):
    """Jacobi::convert_to(Dense): the block-diagonal inverse."""
    d = np.zeros((n, n))
    if prec[0] == "scalar":
        d[np.arange(n), np.arange(n)] = prec[1]
        return d
    _, ptrs, blocks = prec
    for (s, e), blk in zip(zip(ptrs[:-1], ptrs[1:]), blocks):
        d[s:e, s:e] = blk
    return d
