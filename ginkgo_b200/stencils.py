"""Seeded synthetic matrices for the solver workloads (host side, numpy).

Every generator returns CSR arrays ``(row_ptrs int32[n+1], col_idxs int32[nnz],
values float64[nnz])`` with sorted column indices and no duplicates, in the
layout of ``gko::matrix::Csr`` (include/ginkgo/core/matrix/csr.hpp:176-699).
Grids use lexicographic ordering ``i = (z * ny + y) * nx + x`` with Dirichlet
boundaries eliminated, the convention of benchmark/utils/stencil_matrix.hpp.
"""
from __future__ import annotations

import itertools

import numpy as np


def _assemble(n, rows, cols, vals):
    """Sort (row, col) pairs and build CSR (duplicates must not occur)."""
    order = np.lexsort((cols, rows))
    rows = rows[order]
    cols = cols[order].astype(np.int32)
    vals = vals[order].astype(np.float64)
    counts = np.bincount(rows, minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return rp.astype(np.int32), cols, vals


def _grid_stencil(dims, offsets, weights):
    """Assemble a constant-coefficient stencil on a Dirichlet grid.

    ``offsets`` is a list of integer tuples (one per axis, x first) and
    ``weights`` the matching coefficients; neighbours outside the grid are
    dropped (the Dirichlet boundary is eliminated).
    """
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    coords = np.indices(dims[::-1]).reshape(len(dims), -1)[::-1]  # x, y, z
    strides = np.cumprod((1,) + dims[:-1])
    rows_l, cols_l, vals_l = [], [], []
    idx = np.arange(n, dtype=np.int64)
    for off, w in zip(offsets, weights):
        ok = np.ones(n, dtype=bool)
        shift = 0
        for a, o in enumerate(off):
            if o:
                c = coords[a] + o
                ok &= (c >= 0) & (c < dims[a])
                shift += o * int(strides[a])
        r = idx[ok]
        rows_l.append(r)
        cols_l.append(r + shift)
        vals_l.append(np.full(r.shape, w, dtype=np.float64))
    return _assemble(n, np.concatenate(rows_l), np.concatenate(cols_l),
                     np.concatenate(vals_l))


def poisson_2d_5pt(nx: int, ny: int | None = None):
    """2D 5-point Laplacian: 4 on the diagonal, -1 to each grid neighbour."""
    ny = nx if ny is None else ny
    offs = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)]
    return _grid_stencil((nx, ny), offs, [4.0, -1, -1, -1, -1])


def poisson_3d_7pt(nx: int, ny: int | None = None, nz: int | None = None):
    """3D 7-point Laplacian: 6 on the diagonal, -1 to each grid neighbour
    (values of benchmark/utils/stencil_matrix.hpp:206,421)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    offs = [(0, 0, 0)] + [tuple(int(a == i) * s for a in range(3))
                          for i in range(3) for s in (1, -1)]
    return _grid_stencil((nx, ny, nz), offs, [6.0] + [-1.0] * 6)


def anisotropic_27pt(nx: int, coeffs=(1.0, 1e-2, 1e-4)):
    """3D 27-point anisotropic diffusion: the trilinear (Q1) finite-element
    stiffness of -div(diag(cx, cy, cz) grad u) on a uniform grid (scaled by
    the mesh width), Dirichlet boundary eliminated.

    With 1D stiffness S = [-1, 2, -1] and mass M = [1/6, 2/3, 1/6], the
    weight of offset (dx, dy, dz) is
    cx S(dx) M(dy) M(dz) + cy M(dx) S(dy) M(dz) + cz M(dx) M(dy) S(dz).
    The matrix is symmetric positive definite; interior rows have 27 entries,
    boundary rows fewer (nnz = 23,393,656 at 96^3)."""
    S = {-1: -1.0, 0: 2.0, 1: -1.0}
    M = {-1: 1.0 / 6.0, 0: 2.0 / 3.0, 1: 1.0 / 6.0}
    cx, cy, cz = coeffs
    offs, ws = [], []
    for d in itertools.product((-1, 0, 1), repeat=3):
        dx, dy, dz = d
        w = (cx * S[dx] * M[dy] * M[dz] + cy * M[dx] * S[dy] * M[dz]
             + cz * M[dx] * M[dy] * S[dz])
        offs.append(d)
        ws.append(w)
    return _grid_stencil((nx, nx, nx), offs, ws)


def power_law(n: int, seed: int = 0, mu: float = 2.5, sigma: float = 1.0,
              max_len: int = 4096):
    """Random power-law matrix: row lengths round(lognormal(mu, sigma))
    clipped to [1, max_len], columns uniform without duplicates (sorted),
    values ~ N(0, 1)."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.rint(rng.lognormal(mu, sigma, size=n)), 1,
                   min(max_len, n)).astype(np.int64)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    nnz = int(rp[-1])
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, n, size=nnz, dtype=np.int64)
    # resolve duplicates inside a row by redrawing until none are left
    for _ in range(64):
        key = rows * n + cols
        order = np.argsort(key, kind="stable")
        sk = key[order]
        dup = np.zeros(nnz, dtype=bool)
        dup[order[1:][sk[1:] == sk[:-1]]] = True
        nd = int(dup.sum())
        if nd == 0:
            break
        cols[dup] = rng.integers(0, n, size=nd, dtype=np.int64)
    vals = rng.standard_normal(nnz)
    order = np.lexsort((cols, rows))
    return rp.astype(np.int32), cols[order].astype(np.int32), vals[order]


def convection_diffusion_2d(nx: int, ny: int, diffusion: float, vx: float,
                            vy: float):
    """5-point convection-diffusion -d lap(u) + v . grad(u) with unit mesh
    width and central differences: 4d on the diagonal, -d +/- v/2 to the
    neighbours (|v| <= 1 <= 2d keeps the cell Peclet number <= 1)."""
    offs = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)]
    ws = [4.0 * diffusion, -diffusion + 0.5 * vx, -diffusion - 0.5 * vx,
          -diffusion + 0.5 * vy, -diffusion - 0.5 * vy]
    return _grid_stencil((nx, ny), offs, ws)


def most_square_grid(n: int):
    """(nx, ny) with nx * ny == n and nx the largest divisor <= sqrt(n)."""
    a = int(np.floor(np.sqrt(n)))
    while a > 1 and n % a:
        a -= 1
    return n // a, a


def batch_sizes(num_systems: int, lo: int, hi: int, seed: int):
    """System sizes ~ U[lo, hi] (inclusive)."""
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, size=num_systems)


def conductivity_edges(nx: int):
    """Edge list of the 3D 7-point variable-conductivity operator.

    Returns ``(ei, ej)`` (int64): interior edges join grid nodes ``ei`` and
    ``ej``; boundary edges (to the eliminated Dirichlet boundary) have
    ``ej == -1``.  Ordering: interior x-, y-, z-edges, then boundary faces."""
    n = nx ** 3
    idx = np.arange(n, dtype=np.int64).reshape(nx, nx, nx)  # z, y, x
    ei, ej = [], []
    for axis in (2, 1, 0):
        a = np.take(idx, np.arange(nx - 1), axis=axis).ravel()
        b = np.take(idx, np.arange(1, nx), axis=axis).ravel()
        ei.append(a)
        ej.append(b)
    for axis in (2, 1, 0):
        for end in (0, nx - 1):
            a = np.take(idx, [end], axis=axis).ravel()
            ei.append(a)
            ej.append(np.full(a.shape, -1, dtype=np.int64))
    return np.concatenate(ei), np.concatenate(ej)


def conductivity_matrix(nx: int, theta: np.ndarray):
    """A(theta): A_ij = A_ji = -theta_e for an interior edge e = (i, j),
    A_ii = sum of theta over the edges at i (boundary edges included)."""
    n = nx ** 3
    ei, ej = conductivity_edges(nx)
    theta = np.asarray(theta, dtype=np.float64)
    diag = np.bincount(ei, weights=theta, minlength=n)
    inner = ej >= 0
    diag += np.bincount(ej[inner], weights=theta[inner], minlength=n)
    rows = np.concatenate([np.arange(n), ei[inner], ej[inner]])
    cols = np.concatenate([np.arange(n), ej[inner], ei[inner]])
    vals = np.concatenate([diag, -theta[inner], -theta[inner]])
    return _assemble(n, rows, cols, vals)


def std_uniform(seed: int, n: int, lo: float, hi: float):
    """The values std::mt19937(seed) + std::uniform_real_distribution<double>
    (lo, hi) produce with libstdc++: two 32-bit outputs per value combined
    as in generate_canonical<double, 53>.  numpy's legacy RandomState seeds
    MT19937 the same way std::mt19937 does for a 32-bit integer seed."""
    w = np.frombuffer(np.random.RandomState(seed).bytes(8 * n), "<u4")
    w = w.astype(np.float64).reshape(n, 2)
    r = (w[:, 0] + w[:, 1] * 2.0 ** 32) / 2.0 ** 64
    r = np.where(r >= 1.0, np.nextafter(1.0, 0.0), r)
    return r * (hi - lo) + lo
