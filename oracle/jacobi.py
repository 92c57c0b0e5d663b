"""Pure-Python restatement of the reference's block Jacobi preconditioner
(core/preconditioner/jacobi.cpp with reference/preconditioner/
jacobi_kernels.cpp) — TEST INFRASTRUCTURE ONLY.

The checker for a future device block Jacobi: block detection (natural
blocks of rows with equal patterns, then supervariable agglomeration under
max_block_size), extraction and in-place Gauss-Jordan inversion with partial
pivoting of each diagonal block, its application (plain and alpha D^-1 b +
beta x), transposition, conversion to dense, scalar Jacobi, and the L1
modifications, and adaptive-precision block storage (the block
conditioning, the per-group choice of a storage precision and the blocks
rounded to it: generate_adaptive).  Pinned by the reference's own tests
(reference/test/preconditioner/jacobi_kernels.cpp).  Only tests import this
module.

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


def _gauss_jordan(blk):
    """The in-place part of invert_block: returns (b, perm, ok) with b the
    eliminated block before permute_and_transpose_block and ok False when a
    zero pivot ended the elimination."""
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
            return b, perm, False
        for i in range(n):
            b[i, k] = dt(b[i, k] / -d)
        b[k, k] = 0
        for i in range(n):
            for j in range(n):
                b[i, j] = dt(b[i, j] + b[i, k] * b[k, j])
        for j in range(n):
            b[k, j] = dt(b[k, j] / d)
        b[k, k] = dt(1 / d)
    return b, perm, True


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


# ------------------------------------------------------------------------
# Adaptive precision (Jacobi's storage_optimization = autodetect):
# reference/preconditioner/jacobi_kernels.cpp:280-400 (generate,
# validate_precision_reduction_feasibility), core/preconditioner/
# jacobi_utils.hpp (get_supported_storage_reductions,
# get_optimal_storage_reduction, the precision of each encoding).
# Encodings are precision_reduction's byte: (preserving << 4) | nonpreserving,
# 0xff = autodetect.

AUTODETECT = 0xFF
P00, P01, P02, P10, P11, P20 = 0x00, 0x01, 0x02, 0x10, 0x11, 0x20
# precision_reduction_descriptor bits
D00, D02, D11, D20, D01, D10 = 0x00, 0x01, 0x02, 0x04, 0x08, 0x10
_SINGLETON = {P00: D00, P01: D01, P02: D02, P10: D10, P11: D11, P20: D20}


def _half_of_float(f):
    """gko::half's conversion of an FP32 value (round to nearest even, values
    below the smallest normal half flushed to a signed zero)."""
    f = np.asarray(f, np.float32)
    h = f.astype(np.float16)
    small = (np.abs(f) < np.float32(2.0 ** -14)) & np.isfinite(f)
    return np.where(small, np.copysign(np.float16(0), f), h)


def _trunc(x, float_dtype, keep_bits):
    """truncated<T, N>: the top keep_bits bits of each T value."""
    x = np.asarray(x, float_dtype)
    if float_dtype == np.float64:
        u = x.view(np.uint64)
        mask = np.uint64(((1 << keep_bits) - 1) << (64 - keep_bits))
        return (u & mask).view(np.float64)
    u = x.view(np.uint32)
    mask = np.uint32(((1 << keep_bits) - 1) << (32 - keep_bits))
    return (u & mask).view(np.float32)


def storage_roundtrip(x, prec, dtype):
    """Values of dtype (FP64 or FP32) stored at precision encoding prec and
    read back (GKO_PRECONDITIONER_JACOBI_RESOLVE_PRECISION's types)."""
    x = np.asarray(x, dtype)
    if prec == P00:
        return x.copy()
    if dtype == np.float64:
        if prec == P01:
            return x.astype(np.float32).astype(np.float64)
        if prec == P02:
            return _half_of_float(x.astype(np.float32)).astype(np.float64)
        if prec == P10:
            return _trunc(x, np.float64, 32)
        if prec == P11:
            return _trunc(x.astype(np.float32), np.float32, 16).astype(np.float64)
        if prec == P20:
            return _trunc(x, np.float64, 16)
    else:
        if prec in (P01, P02, P11):
            return _half_of_float(x).astype(np.float32)
        if prec in (P10, P20):
            return _trunc(x, np.float32, 16)
    raise ValueError(prec)


def storage_bytes(prec, dtype):
    """Bytes per value of the storage type of encoding prec."""
    if prec == P00:
        return np.dtype(dtype).itemsize
    if dtype == np.float64:
        return {P01: 4, P02: 2, P10: 4, P11: 2, P20: 2}[prec]
    return 2


def _eps(dtype):
    """float_traits eps of each storage type, keyed like storage types:
    (t2t, tr, rr, t, r) = truncate<truncate<T>>, truncate<reduce<T>>,
    reduce<reduce<T>>, truncate<T>, reduce<T>."""
    if dtype == np.float64:
        return (2.0 ** -4, 2.0 ** -7, 2.0 ** -11, 2.0 ** -20, 2.0 ** -24)
    return (2.0 ** -7, 2.0 ** -11, 2.0 ** -11, 2.0 ** -7, 2.0 ** -11)


def _inf_norm(b):
    """compute_inf_norm: the largest absolute row sum (in the block type)."""
    dt = b.dtype.type
    best = dt(0)
    for row in b:
        s = dt(0)
        for v in row:
            s = dt(s + abs(v))
        best = max(best, s)
    return best


def feasible(eliminated, prec, dtype):
    """validate_precision_reduction_feasibility: the eliminated block rounded
    to the storage type and back stays invertible and well conditioned
    (cond >= 1 and cond * eps(dtype) < 1e-3)."""
    dt = np.dtype(dtype).type
    with np.errstate(all="ignore"):  # overflow to inf is part of the check
        tmp = storage_roundtrip(eliminated, prec, dtype).astype(dtype)
        cond = _inf_norm(tmp)
        inv, _, ok = _gauss_jordan(tmp)
        if not ok:
            return False
        cond = dt(cond * _inf_norm(inv))
    eps = np.finfo(dtype).eps / 2  # float_traits eps: 2^-53 / 2^-24
    return bool(cond >= 1.0 and cond * dt(eps) < dt(1e-3))


def supported_reductions(accuracy, cond, ver1, ver2, dtype):
    """get_supported_storage_reductions: the descriptor bits of the
    reductions accurate enough for cond; ver1 / ver2 check the one- and
    two-step non-preserving reductions, each called at most once."""
    dt = np.dtype(dtype).type
    e_t2t, e_tr, e_rr, e_t, e_r = _eps(dtype)
    accurate = lambda e: bool(dt(cond * dt(e)) < dt(accuracy))
    verified1 = 2
    sup = D00
    if accurate(e_t2t):
        sup |= D20
    if accurate(e_tr):
        verified1 = 1 if ver1() else 0
        if verified1:
            sup |= D11
    if accurate(e_rr) and verified1 != 0 and ver2():
        sup |= D02
    if accurate(e_t):
        sup |= D10
    if accurate(e_r):
        if verified1 == 2:
            verified1 = 1 if ver1() else 0
        if verified1 == 1:
            sup |= D01
    return sup


def optimal_reduction(sup):
    """get_optimal_storage_reduction."""
    for bit, prec in ((D02, P02), (D11, P11), (D20, P20), (D01, P01), (D10, P10)):
        if sup & bit:
            return prec
    return P00


def generate_adaptive(rp, ci, v, max_block_size, block_ptrs=None, accuracy=1e-1,
                      precisions=None, aggregate_l1=False, dtype=np.float64):
    """Jacobi::generate with storage_optimization: precisions is None
    (autodetect for every block), one encoding for all blocks, or one per
    block (AUTODETECT where the choice is left to the conditioning).  Blocks
    of one storage group (32 / pow2ceil(max_block_size) blocks) share the
    most reduced precision all of them support.  Returns ("block", ptrs,
    [inverses rounded to their storage and read back], precisions per block,
    conditioning per block)."""
    v = np.asarray(v, dtype=dtype)
    ptrs = list(block_ptrs) if block_ptrs is not None else find_blocks(rp, ci, max_block_size)
    if aggregate_l1:
        rp, ci, v = _with_diagonal(rp, ci, v)
        v = block_l1(rp, ci, v, ptrs).astype(dtype)
    nb = len(ptrs) - 1
    if precisions is None:
        req = [AUTODETECT] * nb
    elif np.isscalar(precisions):
        req = [int(precisions)] * nb
    else:
        req = [int(p) for p in precisions]
    p2 = 1
    while p2 < max_block_size:
        p2 *= 2
    gs = 32 // p2
    dt = np.dtype(dtype).type
    red1 = P01  # reduce<T>
    red2 = P02  # reduce<reduce<T>>
    elim, perms, conds, descs = [], [], [], []
    for b in range(nb):
        s0, e0 = ptrs[b], ptrs[b + 1]
        blk = extract_block(rp, ci, v, s0, e0 - s0, dtype)
        cond = _inf_norm(blk)
        el, perm, _ = _gauss_jordan(blk)
        cond = dt(cond * _inf_norm(el))
        conds.append(cond)
        elim.append(el)
        perms.append(perm)
        if req[b] == AUTODETECT:
            descs.append(supported_reductions(
                accuracy, cond, lambda el=el: feasible(el, red1, dtype),
                lambda el=el: feasible(el, red2, dtype), dtype))
        else:
            descs.append(_SINGLETON.get(req[b], D00))
    chosen = [P00] * nb
    for g0 in range(0, nb, gs):
        acc = 0xFFFFFFFF
        for b in range(g0, min(g0 + gs, nb)):
            acc &= descs[b]
        p = optimal_reduction(acc)
        for b in range(g0, min(g0 + gs, nb)):
            chosen[b] = p
    blocks = []
    for b in range(nb):
        el, perm = elim[b], perms[b]
        n = el.shape[0]
        inv = np.zeros_like(el)
        for i in range(n):
            for j in range(n):
                inv[i, perm[j]] = el[i, j]
        blocks.append(storage_roundtrip(inv, chosen[b], dtype).astype(dtype))
    return ("block", ptrs, blocks), chosen, conds
