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


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 arrays (wrap-around arithmetic)."""
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def banded_rowmajor(n: int, k: int, d: float, dist: int = 1, seed: int = 0, rows_per_chunk: int = 1 << 16):
    """Row-major band ((2k+1) values per row, A(i, j) at i*(2k+1) + k + j - i)
    of the seeded counter-based banded generator: every off-diagonal (i, j)
    with |i - j| <= k inside the matrix is drawn from a hash of (seed, i, j),
    U[-1, 1] (dist 1) or N(0, 1) by Box-Muller (dist 2); the diagonal is
    d * sum_j |A(i, j)|.  The same matrix as the library's
    sap_generate_band_host with these arguments: value for value for dist 1;
    for dist 2 up to the last-bit rounding of numpy's log and cos against the C
    library's."""
    if dist not in (1, 2):
        raise ValueError("dist must be 1 (uniform) or 2 (normal)")
    sw = 2 * k + 1
    out = np.zeros((n, sw))
    s0 = _splitmix64(np.array([np.uint64(seed) ^ np.uint64(0x5A5A5A5A12345678)], dtype=np.uint64))[0]
    offs = np.arange(-k, k + 1, dtype=np.int64)
    for r0 in range(0, n, rows_per_chunk):
        r = np.arange(r0, min(n, r0 + rows_per_chunk), dtype=np.int64)
        c = r[:, None] + offs[None, :]
        ok = (c >= 0) & (c < n) & (offs[None, :] != 0)
        key = (r[:, None].astype(np.uint64) << np.uint64(32)) | (c.astype(np.uint64) & np.uint64(0xFFFFFFFF))
        h = _splitmix64(s0 ^ _splitmix64(key))
        u = (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        if dist == 1:
            val = -1.0 + 2.0 * u
        else:
            u2 = (_splitmix64(h) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            u1 = np.maximum(u, 1e-300)
            val = np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
        val = np.where(ok, val, 0.0)
        # the diagonal sums |off-diagonals| in column order, as the generator does
        rs = np.zeros(len(r))
        for j in range(sw):
            rs += np.abs(val[:, j])
        val[:, k] = d * rs
        out[r0:r0 + len(r)] = val
    return out


def csr_matvec(rp, ci, v, x):
    """y = A x for a CSR matrix (numpy)."""
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    return np.bincount(rows, weights=v * x[ci], minlength=rp.size - 1)
