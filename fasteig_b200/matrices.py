"""Seeded synthetic sparse symmetric matrices for the benchmark shapes.

All generators return host CSR arrays ``(n, rowptr int32, colind int32,
values float64)`` with full symmetric storage and columns sorted within each
row, i.e. the layout ``fasteig_problem::build_csr_from_sparse_matrix``
produces (src/fasteig_problem.cpp:554-607). Grids use natural (x fastest)
ordering, h = 1 and Dirichlet boundaries. The potential draws use
``numpy.random.Generator(PCG64(seed))``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class HostCsr:
    n: int
    rowptr: np.ndarray
    colind: np.ndarray
    values: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.values.size)


def _stencil_csr(dims, offsets, offdiag_fn, diag) -> HostCsr:
    """Assemble a structured-grid operator. ``offsets`` are integer grid shifts
    (excluding 0); ``offdiag_fn(i, j)`` returns the value for neighbour pairs
    (arrays of row and column indices); ``diag`` is an n-vector."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    coords = np.indices(dims[::-1]).reshape(len(dims), -1)[::-1]  # coords[0] = x (fastest)
    strides = [1]
    for d in dims[:-1]:
        strides.append(strides[-1] * d)
    rows_l, cols_l, vals_l = [np.arange(n, dtype=np.int64)], [np.arange(n, dtype=np.int64)], [diag]
    base = np.arange(n, dtype=np.int64)
    for off in offsets:
        ok = np.ones(n, dtype=bool)
        shift = 0
        for ax, o in enumerate(off):
            c = coords[ax] + o
            ok &= (c >= 0) & (c < dims[ax])
            shift += o * strides[ax]
        r = base[ok]
        c = r + shift
        rows_l.append(r)
        cols_l.append(c)
        vals_l.append(offdiag_fn(r, c))
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    vals = np.concatenate(vals_l)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    return HostCsr(n, rowptr.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64))


def _offsets(dim: int, kind: str):
    if kind == "star1":  # 5-point (2D) / 7-point (3D)
        out = []
        for ax in range(dim):
            for s in (-1, 1):
                o = [0] * dim
                o[ax] = s
                out.append(tuple(o))
        return out
    if kind == "star2":  # 13-point (3D): +-1 and +-2 along each axis
        out = []
        for ax in range(dim):
            for s in (-2, -1, 1, 2):
                o = [0] * dim
                o[ax] = s
                out.append(tuple(o))
        return out
    if kind == "box":  # 27-point (3D)
        import itertools
        return [o for o in itertools.product((-1, 0, 1), repeat=dim) if any(o)]
    raise ValueError(kind)


def laplacian_uniform_potential(side: int, dim: int = 3, seed: int = 0) -> HostCsr:
    """3D 7-point (or 2D 5-point) Dirichlet Laplacian (diag 2*dim, off -1) plus a
    diagonal potential drawn uniform[0,1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = side ** dim
    v = rng.random(n)
    return _stencil_csr((side,) * dim, _offsets(dim, "star1"),
                        lambda r, c: np.full(r.size, -1.0), 2.0 * dim + v)


def gaussian_wells(side: int, wells: int = 32, seed: int = 0) -> np.ndarray:
    """Potential V(x) = sum_k -a_k exp(-|x - c_k|^2 / (2 w_k^2)), a_k ~ U[1,5],
    w_k ~ U[2,6] grid units, centres uniform in the box."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.uniform(1.0, 5.0, wells)
    w = rng.uniform(2.0, 6.0, wells)
    c = rng.uniform(0.0, side - 1.0, (wells, 3))
    x = np.arange(side, dtype=np.float64)
    V = np.zeros((side, side, side))  # indexed [z, y, x]
    for k in range(wells):
        gx = np.exp(-(x - c[k, 0]) ** 2 / (2 * w[k] ** 2))
        gy = np.exp(-(x - c[k, 1]) ** 2 / (2 * w[k] ** 2))
        gz = np.exp(-(x - c[k, 2]) ** 2 / (2 * w[k] ** 2))
        V -= a[k] * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return V.reshape(-1)


def laplacian_wells(side: int, wells: int = 32, seed: int = 0, stencil: str = "star1") -> HostCsr:
    """3D 7-point (stencil='star1') or 13-point ('star2') Laplacian plus Gaussian wells."""
    V = gaussian_wells(side, wells, seed)
    offs = _offsets(3, stencil)
    if stencil == "star1":
        return _stencil_csr((side,) * 3, offs, lambda r, c: np.full(r.size, -1.0), 6.0 + V)
    # fourth-order 13-point: (-1/12, 4/3, -5/2, 4/3, -1/12) per axis, negated
    def off(r, c):
        d = np.abs(c - r)
        far = (d == 2) | (d == 2 * side) | (d == 2 * side * side)
        return np.where(far, 1.0 / 12.0, -4.0 / 3.0)
    return _stencil_csr((side,) * 3, offs, off, 3 * 2.5 + V)


def stiffness_mass_27pt(side: int, seed: int = 0):
    """Generalized pair (K, M): K 27-point with K_ij = -(c_i + c_j)/2 for neighbours,
    c ~ LogNormal(0, 0.5) per node, K_ii = sum_j |K_ij| + 1e-3; M = M1 x M1 x M1 with
    M1 = tridiag(1/6, 2/3, 1/6)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = side ** 3
    cnode = rng.lognormal(0.0, 0.5, n)
    offs = _offsets(3, "box")
    K = _stencil_csr((side,) * 3, offs, lambda r, c: -(cnode[r] + cnode[c]) / 2.0, np.zeros(n))
    # diagonal = row sum of |offdiag| + 1e-3
    rows = np.repeat(np.arange(n), np.diff(K.rowptr))
    isdiag = K.colind == rows
    rs = np.zeros(n)
    np.add.at(rs, rows[~isdiag], np.abs(K.values[~isdiag]))
    K.values[isdiag] = rs + 1e-3
    m1 = {-1: 1.0 / 6.0, 0: 2.0 / 3.0, 1: 1.0 / 6.0}

    def mval(r, c):
        out = np.ones(r.size)
        for s in (1, side, side * side):
            dr = (c // s) % side - (r // s) % side
            out *= np.vectorize(m1.get)(dr) if r.size < 16 else np.where(dr == 0, 2.0 / 3.0, 1.0 / 6.0)
        return out
    M = _stencil_csr((side,) * 3, offs, mval, np.full(n, (2.0 / 3.0) ** 3))
    return K, M


def batch_2d_problems(count: int = 512, n_min: int = 4096, n_max: int = 262144, seed: int = 0):
    """Batch of 2D 5-point + U[0,1) problems: n log-uniform in [n_min, n_max], square
    grids of side round(sqrt(n)), nev drawn from {8, 16, 32}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), count))
    sides = np.maximum(2, np.rint(np.sqrt(ns)).astype(int))
    nevs = rng.choice([8, 16, 32], count)
    seeds = rng.integers(0, 2**31 - 1, count)
    return [(laplacian_uniform_potential(int(s), 2, int(sd)), int(k))
            for s, k, sd in zip(sides, nevs, seeds)]
