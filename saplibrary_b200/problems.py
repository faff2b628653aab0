"""Seeded synthetic problems of the benchmark configurations (host, numpy).

All generators are deterministic for a given seed and return CSR arrays
(int32 row offsets, int32 column indices sorted within each row, float64
values) or a row-major band.
"""
from __future__ import annotations

import numpy as np


def convection_diffusion_csr(m: int = 1000, conv: float = 0.3, fill_per_row: int = 2, fill_reach: int = 5000,
                             fill_mag: float = 0.1, seed: int = 0, permute_rows: bool = True):
    """m x m grid, 5-point operator  -Laplace(u) + c . grad(u)  with diffusion 1
    and first-order upwinded convection c = (conv, conv) (unit spacing,
    Dirichlet boundary), plus `fill_per_row` entries per row at distinct
    random columns within +-fill_reach of the diagonal with values
    U[-fill_mag, fill_mag]; the rows are then permuted by a random
    permutation.  Returns (row_offsets, column_indices, values, row_perm),
    row i of the unpermuted matrix being row row_perm[i] of the result."""
    rng = np.random.default_rng(seed)
    n = m * m
    r = np.arange(n, dtype=np.int64)
    gi, gj = r // m, r % m
    rows, cols, vals = [r], [r], [np.full(n, 4.0 + 2.0 * conv)]
    for di, dj, v in ((0, -1, -1.0 - conv), (-1, 0, -1.0 - conv), (0, 1, -1.0), (1, 0, -1.0)):
        ok = (gi + di >= 0) & (gi + di < m) & (gj + dj >= 0) & (gj + dj < m)
        rows.append(r[ok])
        cols.append(r[ok] + di * m + dj)
        vals.append(np.full(int(ok.sum()), v))
    # random fill: distinct columns per row, none on an existing stencil entry
    stencil_offsets = np.array([0, -1, 1, -m, m])
    fill_cols = np.empty((n, fill_per_row), dtype=np.int64)
    for k in range(fill_per_row):
        pending = np.arange(n)
        while pending.size:
            d = rng.integers(-fill_reach, fill_reach + 1, size=pending.size)
            c = pending + d
            bad = (c < 0) | (c >= n) | np.isin(d, stencil_offsets)
            for kk in range(k):
                bad |= c == fill_cols[pending, kk]
            fill_cols[pending[~bad], k] = c[~bad]
            pending = pending[bad]
    rows.append(np.repeat(r, fill_per_row))
    cols.append(fill_cols.ravel())
    vals.append(rng.uniform(-fill_mag, fill_mag, size=n * fill_per_row))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    perm = rng.permutation(n) if permute_rows else np.arange(n)
    rows = perm[rows]
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))])
    return rp.astype(np.int32), cols.astype(np.int32), vals, perm


def csr_matvec(rp, ci, v, x):
    """y = A x for a CSR matrix (numpy)."""
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    return np.bincount(rows, weights=v * x[ci], minlength=rp.size - 1)
