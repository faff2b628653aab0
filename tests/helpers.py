"""Shared test inputs: the reference's synthetic matrices, rebuilt
deterministically (driver_unit_test.cu GetBandedMatrix / GetRhsVector, and
the banded generator of the library)."""
import ctypes

import numpy as np


def unit_test_csr(N=10000, k=20, d=1.0):
    """The matrix of examples/unit_test/driver_unit_test.cu:112-145: glibc
    rand() from its default seed, RAND(L,H) = L + (H-L)*(float)rand()/(float)RAND_MAX,
    diagonal d * sum |off-diagonals|; CSR sorted by row."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    rmax = float(np.float32(2147483647))
    nnz_row = [min(N - 1, i + k) - max(0, i - k) + 1 for i in range(N)]
    rp = np.zeros(N + 1, np.int64)
    rp[1:] = np.cumsum(nnz_row)
    ci = np.empty(rp[-1], np.int32)
    v = np.empty(rp[-1], np.float64)
    pos = 0
    for ir in range(N):
        left, right = max(0, ir - k), min(N - 1, ir + k)
        row_sum = 0.0
        dpos = -1
        for ic in range(left, right + 1):
            val = -10.0 + (20.0 * float(np.float32(libc.rand()))) / rmax
            if ic == ir:
                dpos = pos
            else:
                row_sum += abs(val)
            ci[pos] = ic
            v[pos] = val
            pos += 1
        v[dpos] = d * row_sum
    return rp.astype(np.int32), ci, v


def unit_test_rhs(rp, ci, v):
    """GetRhsVector (driver_unit_test.cu:155-176): x(t) = 400 t (1-t), b = A x."""
    N = rp.size - 1
    t = np.arange(N) / (N - 1)
    x = 400.0 * t * (1.0 - t)
    b = np.zeros(N)
    rows = np.repeat(np.arange(N), np.diff(rp))
    np.add.at(b, rows, v * x[ci])
    return b, x


def band_to_scipy(band, n, K):
    """Row-major band -> scipy.linalg.solve_banded (2K+1, n) storage."""
    A = band.reshape(n, 2 * K + 1)
    ab = np.zeros((2 * K + 1, n))
    for off in range(-K, K + 1):  # column j = i + off
        i = np.arange(max(0, -off), min(n, n - off))
        ab[K - off, i + off] = A[i, K + off]
    return ab


def band_to_dense(band, n, K):
    A = band.reshape(n, 2 * K + 1)
    D = np.zeros((n, n))
    for off in range(-K, K + 1):
        i = np.arange(max(0, -off), min(n, n - off))
        D[i, i + off] = A[i, K + off]
    return D


def band_to_csr(band, n, K):
    D = band.reshape(n, 2 * K + 1)
    rows, cols, vals = [], [], []
    for off in range(-K, K + 1):
        i = np.arange(max(0, -off), min(n, n - off))
        rows.append(i)
        cols.append(i + off)
        vals.append(D[i, K + off])
    rows = np.concatenate(rows); cols = np.concatenate(cols); vals = np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp).astype(np.int32), cols.astype(np.int32), vals


def spd_band(n, K, seed):
    """Row-major band (n x (2K+1)) of a symmetric, strictly diagonally
    dominant matrix with a positive diagonal (hence SPD)."""
    rng = np.random.default_rng(seed)
    band = np.zeros((n, 2 * K + 1))
    for d in range(1, K + 1):
        vals = rng.uniform(-1.0, 1.0, n - d)
        band[: n - d, K + d] = vals   # A(i, i+d)
        band[d:, K - d] = vals        # A(i+d, i)
    band[:, K] = 1.2 * np.abs(band).sum(axis=1)
    return band.ravel()
