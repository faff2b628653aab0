"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: integers (sizes, half-bandwidth, partition count) bit-exact;
preconditioner applies within 1e-10 (FP64 preconditioner) and 2e-4 (FP32
preconditioner) relative 2-norm, since the chunked sweeps and the
factorisation order their FP operations differently from the serial
restatement; FP64 solves to the reference's criterion
||b - A x|| <= relTol ||b|| with the same monitor code.
"""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle
import saplibrary_b200 as sap
from tests.helpers import band_to_csr, band_to_scipy, unit_test_csr, unit_test_rhs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

APPLY_TOL = {"double": 1e-10, "float": 2e-4}


def banded_opts(fact=sap.LU_UL, ptype=sap.Spike, safe=False, relTol=1e-10):
    # the banded preset of examples/synthetic_banded/driver_banded.cu:166-170
    return sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=fact,
                       precondType=ptype, safeFactorization=safe, relTol=relTol, maxNumIterations=100,
                       trackReordering=False)


def setup_pair(band, n, K, P, dtype, fact=sap.LU_UL, ptype=sap.Spike, safe=False):
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, banded_opts(fact, ptype, safe), prec=dtype)
    s.setup(A)
    o = oracle.Precond(P, fact=fact, ptype=ptype, safe=safe, dtype=dtype)
    assert o.setup_banded(band, n, K) == 0
    return A, s, o


def apply_gpu(s, v):
    vd = torch.tensor(v, device="cuda", dtype=torch.float64)
    zd = torch.empty_like(vd)
    s.precond(vd, zd)
    return zd.cpu().numpy()


APPLY_CASES = [  # n, K, P, d, dist, fact
    (20000, 10, 4, 1.0, 1, sap.LU_UL),
    (30011, 50, 10, 1.0, 1, sap.LU_UL),    # ragged partitions, config-0 bandwidth
    (12000, 8, 6, 0.8, 2, sap.LU_UL),
    (15000, 33, 5, 1.0, 0, sap.LU_only),
    (9000, 75, 4, 1.0, 1, sap.LU_UL),      # K >= 70: boosting kernels
    (40000, 120, 8, 0.8, 2, sap.LU_UL),    # factor window in global memory (FP64)
    (5000, 20, 1, 1.0, 1, sap.LU_UL),      # single partition
]


@pytest.mark.parametrize("dtype", ["double", "float"])
@pytest.mark.parametrize("n,K,P,d,dist,fact", APPLY_CASES)
def test_precond_apply_matches_oracle(n, K, P, d, dist, fact, dtype):
    band = sap.generate_band_host(n, K, d, dist, seed=n + K)
    A, s, o = setup_pair(band, n, K, P, dtype, fact)
    assert s.info() == o.info()  # n, K, P after the partition clamp: exact
    rng = np.random.default_rng(K)
    for _ in range(2):
        v = rng.standard_normal(n)
        z = apply_gpu(s, v)
        zo = o.apply(v)
        assert np.all(np.isfinite(z))
        rel = np.linalg.norm(z - zo) / np.linalg.norm(zo)
        assert rel <= APPLY_TOL[dtype], rel


@pytest.mark.parametrize("ptype", [sap.Block, sap.NoPrecond])
def test_block_and_none_preconditioners(ptype):
    n, K, P = 8000, 12, 4
    band = sap.generate_band_host(n, K, 1.0, 1, seed=4)
    A, s, o = setup_pair(band, n, K, P, "double", ptype=ptype)
    v = np.random.default_rng(2).standard_normal(n)
    z, zo = apply_gpu(s, v), o.apply(v)
    assert np.linalg.norm(z - zo) / np.linalg.norm(zo) <= 1e-10


def test_diagonal_matrix_k0():
    n = 1000
    band = sap.generate_band_host(n, 0, 1.0, 1, seed=1)
    band[:] = np.random.default_rng(0).uniform(1.0, 2.0, n)
    A, s, o = setup_pair(band, n, 0, 4, "double")
    v = np.random.default_rng(3).standard_normal(n)
    assert np.allclose(apply_gpu(s, v), v / band, rtol=1e-15)


SOLVE_CASES = [  # n, K, P, d, dist
    (200000, 50, 10, 1.0, 1),  # the config-0 shape
    (60000, 16, 8, 0.9, 2),
    (50000, 100, 16, 1.0, 1),
]


@pytest.mark.parametrize("n,K,P,d,dist", SOLVE_CASES)
def test_fp64_solve_matches_oracle_and_direct(n, K, P, d, dist):
    band = sap.generate_band_host(n, K, d, dist, seed=7)
    xt = np.ones(n)
    b = oracle.spmv_banded(band, n, K, xt)
    A, s, o = setup_pair(band, n, K, P, "double")
    x = np.zeros(n)
    ok = s.solve(sap.MVBanded(A), b, x)  # host buffers through the C ABI
    xo, res = o.solve(b, band=band, K=K, L=2, maxit=100, reltol=1e-10)
    assert ok and res.code == 1
    assert s.getMonitorCode() == res.code and s.getMonitorMessage() == "Converged"
    st = s.getStats()
    assert st.numIterations == res.iterations
    assert st.relResidualNorm <= 1e-10
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) <= 1e-8
    if n <= 60000:
        xd = sl.solve_banded((K, K), band_to_scipy(band, n, K), b)
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) <= 1e-8


def test_device_buffers_solve():
    n, K, P = 40000, 20, 8
    band = sap.generate_band_host(n, K, 1.0, 1, seed=8)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    A, s, o = setup_pair(band, n, K, P, "double")
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros(n, device="cuda", dtype=torch.float64)
    assert s.solve(sap.MVBanded(A), bd, xd)
    assert torch.allclose(xd, torch.ones_like(xd), rtol=0, atol=1e-8)


def test_fp32_preconditioner_matches_oracle_monitor():
    # mixed mode as in the reference: both stop on stagnation near FP32 accuracy
    n, K, P = 30000, 20, 6
    band = sap.generate_band_host(n, K, 1.0, 1, seed=9)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    A, s, o = setup_pair(band, n, K, P, "float")
    x = np.zeros(n)
    s.solve(sap.MVBanded(A), b, x)
    xo, res = o.solve(b, band=band, K=K, L=2, maxit=100, reltol=1e-10)
    assert s.getMonitorCode() == res.code == -3
    assert s.getStats().relResidualNorm < 1e-6


def test_unit_test_config_through_csr():
    # examples/unit_test/driver_unit_test.cu:49-94 with a double preconditioner
    rp, ci, v = unit_test_csr()
    b, xt = unit_test_rhs(rp, ci, v)
    A = sap.CsrMatrix(rp, ci, v)
    opts = sap.Options(trackReordering=False, variableBandwidth=False, factMethod=sap.LU_UL,
                       performReorder=False, applyScaling=False, relTol=1e-13)
    s = sap.Solver(10, opts, prec="double")
    s.setup(A)
    assert s.info() == (10000, 20, 10)
    x = np.zeros(b.size)
    success = s.solve(sap.SpmvCusp(A), b, x)
    assert success
    assert s.getMonitorCode() == 1
    assert s.getMonitorMessage() == "Converged"
    assert s.getStats().relResidualNorm <= 1e-13


def test_spmv_functors_match_oracle():
    n, K = 50000, 30
    band = sap.generate_band_host(n, K, 1.0, 2, seed=10)
    x = np.random.default_rng(5).standard_normal(n)
    A = sap.BandedMatrix.from_array(band, n, K)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    sap.MVBanded(A)(xd, yd)
    yo = oracle.spmv_banded(band, n, K, x)
    assert np.allclose(yd.cpu().numpy(), yo, rtol=1e-13, atol=1e-12)
    rp, ci, v = band_to_csr(band, n, K)
    C = sap.CsrMatrix(rp, ci, v)
    sap.SpmvCusp(C)(xd, yd)
    assert np.allclose(yd.cpu().numpy(), oracle.spmv_csr(rp, ci, v, x), rtol=1e-13, atol=1e-12)


def test_zero_pivot_raises_system_error():
    n, K = 4000, 5
    band = sap.generate_band_host(n, K, 1.0, 1, seed=2).reshape(n, 2 * K + 1)
    band[0, :] = 0.0
    A = sap.BandedMatrix.from_array(band.ravel(), n, K)
    s = sap.Solver(2, banded_opts(), prec="double")
    with pytest.raises(sap.SystemError) as e:
        s.setup(A)
    assert e.value.reason == sap.SystemError.Zero_pivoting
    s2 = sap.Solver(2, banded_opts(safe=True), prec="double")  # boosting instead
    assert s2.setup(A)


def test_illegal_call_order():
    n, K = 2000, 4
    band = sap.generate_band_host(n, K, 1.0, 1, seed=2)
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(2, banded_opts(), prec="double")
    with pytest.raises(sap.SystemError) as e:
        s.solve(sap.MVBanded(A), np.ones(n), np.zeros(n))
    assert e.value.reason == sap.SystemError.Illegal_solve
    with pytest.raises(sap.SystemError) as e:
        s.update(np.ones(3))
    assert e.value.reason == sap.SystemError.Illegal_update


def test_kernels_were_launched():
    before = sap.kernel_launch_count()
    n, K = 3000, 6
    band = sap.generate_band_host(n, K, 1.0, 1, seed=3)
    A, s, o = setup_pair(band, n, K, 3, "double")
    apply_gpu(s, np.ones(n))
    assert sap.kernel_launch_count() > before + 10


@pytest.mark.parametrize("n", [1, 1000, 3_000_001])
def test_blas_dots_match_numpy(n):
    rng = np.random.default_rng(n)
    xs = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(3)]
    ys = [torch.tensor(rng.standard_normal(n), device="cuda") for _ in range(3)]
    out = torch.empty(3, device="cuda", dtype=torch.float64)
    sap.blas_dots(xs, ys, out)
    torch.cuda.synchronize()
    ref = [float(np.dot(x.cpu().numpy(), y.cpu().numpy())) for x, y in zip(xs, ys)]
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)
