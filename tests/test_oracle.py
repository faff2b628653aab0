"""The CPU oracle checked against independent references: scipy's direct
banded LU (LAPACK gbsv), dense numpy products, and the assertions of the
reference's only unit test (examples/unit_test/driver_unit_test.cu:89-93)."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle
import saplibrary_b200 as sap
from tests.helpers import band_to_dense, band_to_scipy, band_to_csr, unit_test_csr, unit_test_rhs

CASES = [  # n, K, P, d, dist, fact
    (2000, 10, 4, 1.0, 1, sap.LU_UL),
    (3001, 8, 5, 0.8, 2, sap.LU_UL),   # ragged partitions, weak dominance
    (4000, 12, 3, 1.0, 1, sap.LU_only),
    (1500, 30, 7, 1.2, 0, sap.LU_UL),
    (900, 75, 4, 1.0, 1, sap.LU_UL),   # K >= 70: boosting kernels
]


@pytest.mark.parametrize("n,K,P,d,dist,fact", CASES)
def test_oracle_fp64_solve_matches_direct(n, K, P, d, dist, fact):
    band = sap.generate_band_host(n, K, d, dist, seed=11)
    xt = np.ones(n)
    b = oracle.spmv_banded(band, n, K, xt)
    pc = oracle.Precond(P, fact=fact, dtype="double")
    assert pc.setup_banded(band, n, K) == 0
    n_, K_, P_ = pc.info()
    assert (n_, K_) == (n, K)
    assert P_ == min(P, max(1, n // max(K + 1, 2 * K)))  # precond.h:2116-2117
    x, res = pc.solve(b, band=band, K=K, L=2, maxit=100, reltol=1e-10)
    xd = sl.solve_banded((K, K), band_to_scipy(band, n, K), b)
    assert res.code == 1
    assert res.rel_res_norm <= 1e-10
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8


@pytest.mark.parametrize("n,K,P,d,dist,fact", CASES[:3])
def test_oracle_fp32_preconditioner_stagnates_at_fp32_accuracy(n, K, P, d, dist, fact):
    # Right preconditioning with the final x = P^-1 xx applied in FP32
    # (bicgstab2.h:316-318) bounds the achievable residual near 1e-7.
    band = sap.generate_band_host(n, K, d, dist, seed=11)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    pc = oracle.Precond(P, fact=fact, dtype="float")
    assert pc.setup_banded(band, n, K) == 0
    x, res = pc.solve(b, band=band, K=K, L=2, maxit=100, reltol=1e-10)
    assert res.code == -3  # "Stagnation encountered"
    assert 1e-9 < res.rel_res_norm < 1e-5


def test_oracle_apply_is_inverse_for_exact_partition():
    # P = 1: the preconditioner is the exact banded LU solve.
    n, K = 600, 9
    band = sap.generate_band_host(n, K, 1.0, 1, seed=3)
    pc = oracle.Precond(1, dtype="double")
    assert pc.setup_banded(band, n, K) == 0
    v = np.random.default_rng(0).standard_normal(n)
    z = pc.apply(v)
    assert np.allclose(band_to_dense(band, n, K) @ z, v, rtol=0, atol=1e-10)


def test_oracle_spmv_matches_dense():
    n, K = 300, 7
    band = sap.generate_band_host(n, K, 1.0, 2, seed=5)
    x = np.random.default_rng(1).standard_normal(n)
    y = oracle.spmv_banded(band, n, K, x)
    assert np.allclose(y, band_to_dense(band, n, K) @ x, rtol=1e-13, atol=1e-12)
    rp, ci, v = band_to_csr(band, n, K)
    assert np.allclose(oracle.spmv_csr(rp, ci, v, x), y, rtol=1e-13, atol=1e-12)


def test_oracle_zero_pivot_is_reported():
    # K < 70, no safe factorization: a zero pivot raises Zero_pivoting
    # (precond.h:4404-4405).
    n, K = 400, 5
    band = sap.generate_band_host(n, K, 1.0, 1, seed=2).reshape(n, 2 * K + 1)
    band[0, :] = 0.0  # first row zero -> first pivot zero
    pc = oracle.Precond(2, dtype="double")
    assert pc.setup_banded(band.ravel(), n, K) == -1
    pcs = oracle.Precond(2, dtype="double", safe=True)  # boosting instead
    assert pcs.setup_banded(band.ravel(), n, K) == 0


@pytest.fixture(scope="module")
def unit_test_problem():
    rp, ci, v = unit_test_csr()
    b, x = unit_test_rhs(rp, ci, v)
    return rp, ci, v, b, x


def test_unit_test_assertions_double_preconditioner(unit_test_problem):
    # driver_unit_test.cu:49-94: N=1e4, K=20, P=10, d=1, LU_UL, relTol=1e-13.
    rp, ci, v, b, xt = unit_test_problem
    pc = oracle.Precond(10, fact=sap.LU_UL, dtype="double")
    assert pc.setup_csr(rp.size - 1, rp, ci, v) == 0
    assert pc.info() == (10000, 20, 10)
    x, res = pc.solve(b, csr=(rp, ci, v), L=2, maxit=100, reltol=1e-13)
    assert res.code == 1                      # EXPECT_EQ(1, getMonitorCode())
    assert res.rel_res_norm <= 1e-13          # EXPECT_GE(1e-13, relResidualNorm)
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-12


def test_unit_test_float_preconditioner_stagnates(unit_test_problem):
    # The same test with PREC_REAL=float (driver_unit_test.cu:27-28) stops on
    # stagnation near FP32 accuracy in this restatement.
    rp, ci, v, b, xt = unit_test_problem
    pc = oracle.Precond(10, fact=sap.LU_UL, dtype="float")
    assert pc.setup_csr(rp.size - 1, rp, ci, v) == 0
    x, res = pc.solve(b, csr=(rp, ci, v), L=2, maxit=100, reltol=1e-13)
    assert res.code == -3
    assert res.rel_res_norm < 1e-6


def test_oracle_classic_bicgstab_and_minres_converge():
    from tests.helpers import spd_band
    n, K, P = 3000, 6, 3
    band = spd_band(n, K, seed=3)
    xt = np.linspace(1.0, 2.0, n)
    b = oracle.spmv_banded(band, n, K, xt)
    for L in (0, -1):
        o = oracle.Precond(P, fact=1, ptype=1, dtype="double")
        assert o.setup_banded(band, n, K) == 0
        x, res = o.solve(b, band=band, K=K, L=L, maxit=200, reltol=1e-10)
        assert res.code > 0, (L, res.code)
        assert np.linalg.norm(x - xt) / np.linalg.norm(xt) <= 1e-8


def test_mlp_oracle_gradient_matches_central_differences():
    from oracle import mlp_oracle
    rng = np.random.default_rng(2)
    shape = (16, 8, 8, 7)
    n = 8 * 16 + 8 + 8 * 8 + 8 + 7 * 8 + 7
    p = rng.standard_normal(n) * 0.3
    X = rng.standard_normal((30, 16))
    y = rng.integers(0, 7, 30)
    _, g = mlp_oracle.loss_and_grad(p, shape, X, y)
    for k in range(0, n, 17):
        e = np.zeros(n)
        e[k] = 1e-6
        d = (mlp_oracle.loss_and_grad(p + e, shape, X, y)[0] - mlp_oracle.loss_and_grad(p - e, shape, X, y)[0]) / 2e-6
        assert abs(d - g[k]) <= 1e-6 + 1e-5 * abs(g[k])
