"""The reordering oracle (sap/graph.h restatement) checked against
independent properties: the DB matching is a minimum-cost assignment of the
costs log(rowmax / |a_ij|) (scipy's linear_sum_assignment), the DB scaling
makes the matched entries 1 and every entry <= 1 in magnitude, RCM and
drop-off respect their contracts, and the FP64 sparse solve meets the
stopping criterion and matches scipy's direct solver."""
import numpy as np
import pytest
import scipy.sparse as sps
import scipy.sparse.linalg as spl
from scipy.optimize import linear_sum_assignment

import oracle
from saplibrary_b200.problems import convection_diffusion_csr


def family(m, seed=None):
    return convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m if seed is None else seed)


@pytest.mark.parametrize("m", [12, 20])
def test_db_matching_is_an_optimal_assignment(m):
    rp, ci, v, _ = family(m)
    n = m * m
    sp = oracle.SparsePrecond(1, dtype="double", dropFrac=0.0)
    assert sp.setup(rp, ci, v, factor=False) == 0
    perm = sp.ints("dbRowPerm")
    assert np.array_equal(np.sort(perm), np.arange(n))
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    A[rows, ci] = np.abs(v)
    rowmax = A.max(axis=1)
    with np.errstate(divide="ignore"):
        cost = np.where(A > 0, np.log(rowmax[:, None] / A), 1e30)
    r, c = linear_sum_assignment(cost)
    best = cost[r, c].sum()
    got = cost[np.arange(n), perm].sum()  # row i matched to column perm[i]
    assert got == pytest.approx(best, rel=1e-12, abs=1e-9)


def test_db_scaling_makes_matched_entries_one():
    m = 16
    rp, ci, v, _ = family(m)
    n = m * m
    sp = oracle.SparsePrecond(1, dtype="double", dropFrac=0.0)
    assert sp.setup(rp, ci, v, factor=False) == 0
    rs, cs = sp.reals(0), sp.reals(1)
    perm = sp.ints("dbRowPerm")
    rows = np.repeat(np.arange(n), np.diff(rp))
    scaled = np.abs(v) * rs[rows] * cs[ci]
    assert scaled.max() <= 1.0 + 1e-12
    diag = scaled[ci == perm[rows]]
    assert diag.size == n and np.allclose(diag, 1.0, rtol=1e-12)


@pytest.mark.parametrize("frac", [1e-4, 1e-2])
def test_drop_off_budget_and_bandwidths(frac):
    rp, ci, v, _ = family(40)
    sp = oracle.SparsePrecond(4, dtype="double", dropFrac=frac)
    assert sp.setup(rp, ci, v, factor=False) == 0
    inf = sp.info()
    assert 0 < inf.drop_actual <= frac
    assert inf.K <= inf.k_reorder <= inf.k_db or inf.k_reorder <= inf.k_db
    assert max(sp.ints("ks")) <= inf.K
    for name in ("finalPerm", "finalReordering"):
        assert np.array_equal(np.sort(sp.ints(name)), np.arange(40 * 40))


@pytest.mark.parametrize("m,P", [(30, 4), (60, 8)])
def test_sparse_fp64_solve_matches_direct(m, P):
    rp, ci, v, _ = family(m)
    n = m * m
    b = np.random.default_rng(m).standard_normal(n)
    sp = oracle.SparsePrecond(P, dtype="double", dropFrac=1e-4)
    assert sp.setup(rp, ci, v) == 0
    x, res = sp.solve(b, maxit=100, reltol=1e-10)
    assert res.code == 1 and res.rel_res_norm <= 1e-10
    xd = spl.spsolve(sps.csr_matrix((v, ci, rp), shape=(n, n)).tocsc(), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8
