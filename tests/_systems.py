"""Synthetic linear systems shaped like the film-height matrix I + theta dt J
(13-point fourth-order stencil on interior rows, two-entry mirror rows on the
two ghost layers, diagonal first in storage order), for solver parity at
sizes the committed fixtures do not cover.  Seeded; numpy only."""
from __future__ import annotations

import numpy as np

#  stencil offsets of the 13-point set in storage order (diagonal first)
_OFF = [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1), (-2, 0), (2, 0), (0, -2), (0, 2),
        (-1, -1), (1, -1), (-1, 1), (1, 1)]
_BIH = np.array([20, -8, -8, -8, -8, 1, 1, 1, 1, 2, 2, 2, 2], dtype=np.float64)


def sorted_mirror(rowptr: np.ndarray, col: np.ndarray):
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rowptr))
    order = np.lexsort((col, rows))
    return col[order].astype(np.int32), order.astype(np.int32)


def film_system(N: int, seed: int = 0, stiff: float = 1.0, periodic: bool = False) -> dict:
    """A dump-like dict for an N x N grid with two ghost layers."""
    rng = np.random.default_rng(seed)
    nx = N + 4
    n = nx * nx
    jj, ii = np.divmod(np.arange(n), nx)
    interior = (ii >= 2) & (ii < nx - 2) & (jj >= 2) & (jj < nx - 2)
    mob = 0.5 + rng.random(n)
    rowlen = np.where(interior, 13, 2)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    rowptr[1:] = np.cumsum(rowlen)
    nnz = int(rowptr[-1])
    col = np.empty(nnz, dtype=np.int32)
    val = np.empty(nnz, dtype=np.float64)
    bc = (~interior).astype(np.int32)
    # interior rows
    idx = np.nonzero(interior)[0]
    base = rowptr[idx]
    for q, (dx, dy) in enumerate(_OFF):
        c = (jj[idx] + dy) * nx + (ii[idx] + dx)
        col[base + q] = c
        v = stiff * mob[idx] * _BIH[q] * (1.0 + 0.05 * rng.standard_normal(idx.size))
        if q == 0:
            v = 1.0 + stiff * mob[idx] * _BIH[0]
        val[base + q] = v
    # ghost rows: x_ghost - x_partner = 0 (mirror, or periodic copy)
    g = np.nonzero(~interior)[0]
    gi, gj = ii[g].copy(), jj[g].copy()

    def partner(a):
        if periodic:
            return np.where(a < 2, a + (nx - 4), np.where(a >= nx - 2, a - (nx - 4), a))
        return np.where(a < 2, 3 - a, np.where(a >= nx - 2, 2 * (nx - 2) - 1 - a, a))

    pi, pj = partner(gi), partner(gj)
    gb = rowptr[g]
    col[gb] = g
    val[gb] = 1.0
    col[gb + 1] = pj * nx + pi
    val[gb + 1] = -1.0
    rhs = np.where(interior, rng.standard_normal(n) * 1e-3, 0.0)
    scol, ssrc = sorted_mirror(rowptr, col)
    return {"n": n, "nnz": nnz, "rowptr": rowptr, "col": col, "sorted_col": scol, "sorted_src": ssrc,
            "bc": bc, "values": val, "rhs": rhs, "x0": np.zeros(n), "precondition": 2, "scaling": 1,
            "max_iteration": 8000, "epsilon": 1e-13, "conc": 0, "flavour": 0}


def poisson1d(n: int) -> dict:
    """The 1-D Poisson problem of the reference's test_linear_solver.cpp:38-61
    (u'' = 2 on [-1, 1], u = 0 at both ends through the ghost average),
    built here in the same storage order (diagonal first)."""
    dx = 2.0 / (n - 2)
    rows = [[(0, 0.5), (1, 0.5)]]
    for i in range(1, n - 1):
        rows.append([(i, -2.0 / (dx * dx)), (i - 1, 1.0 / (dx * dx)), (i + 1, 1.0 / (dx * dx))])
    rows.append([(n - 1, 0.5), (n - 2, 0.5)])
    rowptr = np.zeros(n + 1, np.int32)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([c for r in rows for c, _ in r], np.int32)
    val = np.array([v for r in rows for _, v in r], np.float64)
    rhs = np.full(n, 2.0)
    rhs[0] = rhs[-1] = 0.0
    scol, ssrc = sorted_mirror(rowptr, col)
    x_exact = np.array([(-1.0 - 0.5 * dx + i * dx) ** 2 - 1.0 for i in range(n)])
    return {"n": n, "nnz": int(rowptr[-1]), "rowptr": rowptr, "col": col, "sorted_col": scol,
            "sorted_src": ssrc, "values": val, "rhs": rhs, "x0": np.zeros(n), "precondition": 2,
            "scaling": 1, "max_iteration": 10 * n, "epsilon": 1e-13, "conc": 0, "exact": x_exact, "dx": dx}
