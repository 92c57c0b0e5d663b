"""Pure-Python restatement of the reference's sparse matrix products and sums
on Csr (reference/matrix/csr_kernels.cpp: spgemm, advanced_spgemm, spgeam;
reference/components/csr_spgeam.hpp) and of the Hybrid (Ell + Coo) format
with its width strategies (include/ginkgo/core/matrix/hybrid.hpp) — TEST
INFRASTRUCTURE ONLY.

The checker for future device SpGEMM / SpGEAM / Hybrid kernels.  Matrices are Csr
triples (row_ptrs, col_idxs, values); results have sorted columns.  Pinned
by the reference's own tests (reference/test/matrix/csr_kernels.cpp).  Only
tests import this module.
"""
from __future__ import annotations

import numpy as np


def _rows(m):
    rp, ci, v = m
    return [(list(ci[rp[r]:rp[r + 1]]), list(v[rp[r]:rp[r + 1]])) for r in range(len(rp) - 1)]


def _pack(rows, dtype):
    rp = np.zeros(len(rows) + 1, dtype=np.int64)
    rp[1:] = np.cumsum([len(c) for c, _ in rows])
    ci = np.array([c for cols, _ in rows for c in cols], dtype=np.int64)
    v = np.array([x for _, vals in rows for x in vals], dtype=dtype)
    return rp, ci, v


def _accumulate(acc, cols, vals, scale, dt):
    """spgemm_accumulate_row: cols[c] += scale * v, in storage order."""
    for c, x in zip(cols, vals):
        acc[c] = dt(acc.get(c, dt(0)) + dt(scale * x))


def _accumulate2(acc, a_cols, a_vals, b_rows, scale, dt):
    """spgemm_accumulate_row2: cols[b_col] += scale * a_val * b_val over A's
    row entries, then B's row entries, in storage order."""
    for ac, av in zip(a_cols, a_vals):
        bc, bv = b_rows[ac]
        for c, x in zip(bc, bv):
            acc[c] = dt(acc.get(c, dt(0)) + dt(dt(scale * av) * x))


def spgemm(a, b, dtype=np.float64):
    """C = A B (spgemm, csr_kernels.cpp:199-245): the pattern is the union
    of B's rows selected by A's row, columns ascending (an ordered map)."""
    dt = np.dtype(dtype).type
    b_rows = _rows(b)
    out = []
    for cols, vals in _rows(a):
        acc = {}
        _accumulate2(acc, cols, vals, b_rows, dt(1), dt)
        ks = sorted(acc)
        out.append((ks, [acc[k] for k in ks]))
    return _pack(out, dtype)


def advanced_spgemm(alpha, a, b, beta, d, dtype=np.float64):
    """C = alpha A B + beta D (advanced_spgemm, :247-300): D's row first,
    then the product, accumulated into one ordered map per row."""
    dt = np.dtype(dtype).type
    b_rows, d_rows = _rows(b), _rows(d)
    out = []
    for r, (cols, vals) in enumerate(_rows(a)):
        acc = {}
        _accumulate(acc, *d_rows[r], dt(beta), dt)
        _accumulate2(acc, cols, vals, b_rows, dt(alpha), dt)
        ks = sorted(acc)
        out.append((ks, [acc[k] for k in ks]))
    return _pack(out, dtype)


def spgeam(alpha, a, beta, b, dtype=np.float64):
    """C = alpha A + beta B (spgeam, :424-470 with abstract_spgeam,
    csr_spgeam.hpp): a merge of the two sorted rows; every column present in
    either is stored, even where the sum is zero."""
    dt = np.dtype(dtype).type
    out = []
    for (ac, av), (bc, bv) in zip(_rows(a), _rows(b)):
        i = j = 0
        cols, vals = [], []
        while i < len(ac) or j < len(bc):
            ca = ac[i] if i < len(ac) else None
            cb = bc[j] if j < len(bc) else None
            if cb is None or (ca is not None and ca < cb):
                cols.append(ca), vals.append(dt(dt(alpha) * av[i] + dt(beta) * dt(0)))
                i += 1
            elif ca is None or cb < ca:
                cols.append(cb), vals.append(dt(dt(alpha) * dt(0) + dt(beta) * bv[j]))
                j += 1
            else:
                cols.append(ca), vals.append(dt(dt(alpha) * av[i] + dt(beta) * bv[j]))
                i += 1
                j += 1
        out.append((cols, vals))
    return _pack(out, dtype)


# ------------------------------------------------------------- Hybrid ----
# matrix::Hybrid (include/ginkgo/core/matrix/hybrid.hpp): an Ell part of
# `width` entries per row (column-major, stride = rows, padding column -1)
# and a Coo part with the rest of every longer row.

def hybrid_width(row_nnz, strategy="automatic", value_bytes=8, index_bytes=4,
                 num_columns=None, percent=None, ratio=None):
    """compute_ell_num_stored_elements_per_row of the strategies
    (hybrid.hpp:188-360): column_limit(num_columns); imbalance_limit(percent)
    = the sorted row length at floor(rows * percent) (the longest for
    percent >= 1); imbalance_bounded_limit(percent, ratio) = min of that and
    floor(rows * ratio); minimal_storage_limit = imbalance_limit(si / (sv +
    2 si)); automatic = imbalance_bounded_limit(1/3, 0.001)."""
    nnz = sorted(int(x) for x in row_nnz)
    n = len(nnz)

    def imbalance(p):
        p = min(max(p, 0.0), 1.0)
        if n == 0:
            return 0
        return nnz[int(n * p)] if p < 1 else nnz[-1]

    if strategy == "column_limit":
        return int(num_columns)
    if strategy == "imbalance_limit":
        return imbalance(0.8 if percent is None else percent)
    if strategy == "imbalance_bounded_limit":
        p = 0.8 if percent is None else percent
        q = 0.0001 if ratio is None else ratio
        return min(imbalance(p), int(n * q))
    if strategy == "minimal_storage_limit":
        return imbalance(index_bytes / (value_bytes + 2 * index_bytes))
    if strategy == "automatic":
        return min(imbalance(1.0 / 3.0), int(n * 0.001))
    raise ValueError(strategy)


def csr_to_hybrid(rp, ci, v, width):
    """Csr -> Hybrid: the first `width` entries of every row into Ell, the
    rest into Coo in row order (csr::convert_to_hybrid)."""
    n = len(rp) - 1
    ell_c = np.full(width * n, -1, dtype=np.int64)
    ell_v = np.zeros(width * n, dtype=np.asarray(v).dtype)
    coo_r, coo_c, coo_v = [], [], []
    for r in range(n):
        for k, idx in enumerate(range(rp[r], rp[r + 1])):
            if k < width:
                ell_c[k * n + r] = ci[idx]
                ell_v[k * n + r] = v[idx]
            else:
                coo_r.append(r), coo_c.append(ci[idx]), coo_v.append(v[idx])
    return {"rows": n, "width": width, "stride": n, "ell_col_idxs": ell_c,
            "ell_values": ell_v, "coo_row_idxs": np.array(coo_r, dtype=np.int64),
            "coo_col_idxs": np.array(coo_c, dtype=np.int64),
            "coo_values": np.array(coo_v, dtype=ell_v.dtype)}


def hybrid_apply(h, x, alpha=None, beta=None, y=None):
    """y = A x (or alpha A x + beta y): the Ell part row by row over its
    slots, then the Coo entries in order (hybrid::spmv = ell + coo)."""
    x = np.asarray(x)
    x2 = x.reshape(len(x), -1)
    n, w, s = h["rows"], h["width"], h["stride"]
    out = np.zeros((n, x2.shape[1]), dtype=x2.dtype)
    for r in range(n):
        for k in range(w):
            c = h["ell_col_idxs"][k * s + r]
            if c >= 0:
                out[r] += h["ell_values"][k * s + r] * x2[c]
    for r, c, val in zip(h["coo_row_idxs"], h["coo_col_idxs"], h["coo_values"]):
        out[r] += val * x2[c]
    if alpha is not None:
        y2 = np.asarray(y).reshape(out.shape)
        out = alpha * out + (beta * y2 if beta != 0 else 0)
    return out[:, 0] if x.ndim == 1 else out


def hybrid_to_csr(h):
    """Hybrid -> Csr: every row's Ell slots (padding dropped) then its Coo
    entries, columns sorted."""
    n, w, s = h["rows"], h["width"], h["stride"]
    rows = [([], []) for _ in range(n)]
    for r in range(n):
        for k in range(w):
            c = h["ell_col_idxs"][k * s + r]
            if c >= 0:
                rows[r][0].append(int(c)), rows[r][1].append(h["ell_values"][k * s + r])
    for r, c, val in zip(h["coo_row_idxs"], h["coo_col_idxs"], h["coo_values"]):
        rows[r][0].append(int(c)), rows[r][1].append(val)
    out = []
    for cols, vals in rows:
        order = np.argsort(cols, kind="stable")
        out.append(([cols[i] for i in order], [vals[i] for i in order]))
    return _pack(out, h["ell_values"].dtype)
