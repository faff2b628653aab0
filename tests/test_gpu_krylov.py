"""The classic BiCGStab (sap/bicgstab.h:50-155) and MINRES
(sap/minres.h:40-195) drivers on the GPU against the oracle's restatements:
same monitor code and iteration count, relative residual within relTol and
solution within 1e-9 of the oracle's."""
import numpy as np
import pytest

import oracle
import saplibrary_b200 as sap
from tests.helpers import spd_band

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def opts(solver, ptype=sap.Spike, relTol=1e-10):
    return sap.Options(solverType=solver, performReorder=False, variableBandwidth=False, applyScaling=False,
                       factMethod=sap.LU_UL, precondType=ptype, relTol=relTol, maxNumIterations=200)


def run_pair(band, n, K, P, solver, L, ptype=sap.Spike):
    b = oracle.spmv_banded(band, n, K, np.linspace(1.0, 2.0, n))
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, opts(solver, ptype), prec="double")
    s.setup(A)
    x = np.zeros(n)
    s.solve(sap.MVBanded(A), b, x)
    o = oracle.Precond(P, fact=sap.LU_UL, ptype=ptype, dtype="double")
    assert o.setup_banded(band, n, K) == 0
    xo, res = o.solve(b, band=band, K=K, L=L, maxit=200, reltol=1e-10)
    return s, x, xo, res


@pytest.mark.parametrize("n,K,P,d", [(50000, 20, 8, 0.9), (30000, 60, 4, 0.8)])
def test_classic_bicgstab_matches_oracle(n, K, P, d):
    band = sap.generate_band_host(n, K, d, 2, seed=n + K)
    s, x, xo, res = run_pair(band, n, K, P, sap.BiCGStab, 0)
    assert s.getMonitorCode() == res.code == 1
    assert s.getStats().numIterations == res.iterations
    assert s.getStats().relResidualNorm <= 1e-10
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9


@pytest.mark.parametrize("n,K,P", [(40000, 16, 4), (20000, 40, 2)])
def test_minres_matches_oracle_on_spd_band(n, K, P):
    band = spd_band(n, K, seed=n)
    s, x, xo, res = run_pair(band, n, K, P, sap.MINRES, -1, ptype=sap.Block)
    assert s.getMonitorCode() == res.code
    assert s.getMonitorCode() > 0
    assert s.getStats().numIterations == res.iterations
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9


@pytest.mark.parametrize("seed", [0, 1])
def test_csr_spmv_row_blocks_with_empty_and_long_rows(seed):
    # the row-block CSR SpMV: rows of 0 .. 11 entries, empty rows, a few rows
    # longer than one block's entry budget (the CTA-wide branch), ragged sizes
    rng = np.random.default_rng(seed)
    n = 30011
    lens = rng.integers(0, 12, n)
    lens[rng.integers(0, n, 50)] = 0
    lens[rng.integers(0, n, 3)] = 5000 + seed
    lens[-1] = 3000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens]).astype(np.int32)
    v = rng.standard_normal(rp[-1])
    A = sap.CsrMatrix(rp, ci, v)
    x = rng.standard_normal(n)
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    sap.SpmvCusp(A)(torch.tensor(x, device="cuda"), y)
    rows = np.repeat(np.arange(n), lens)
    ref = np.bincount(rows, weights=v * x[ci], minlength=n)
    scale = np.bincount(rows, weights=np.abs(v * x[ci]), minlength=n)
    assert np.all(np.abs(y.cpu().numpy() - ref) <= 1e-14 * scale + 1e-300)
