"""The wide-band block path (half-bandwidth from 256 up by default, and every
band above 1024) against the oracle through the C ABI.

The block path factors each partition as block tridiagonal with dense block
LUs; the factors equal the band LU's up to rounding, so applies are held to
the same relative 2-norm tolerances as the narrow path (1e-10 FP64, 2e-4
FP32 preconditioner) and FP64 solves to the reference's criterion
||b - A x|| <= relTol ||b||.
"""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle
import saplibrary_b200 as sap
from tests.helpers import band_to_scipy
from tests.test_gpu_parity import APPLY_TOL, apply_gpu, setup_pair

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

WIDE_CASES = [  # n, K, P, d, dist, fact, precond type
    (20000, 300, 4, 1.0, 1, sap.LU_UL, sap.Spike),
    (24011, 257, 5, 0.8, 2, sap.LU_only, sap.Spike),  # ragged partitions, padded last block
    (7000, 300, 1, 1.0, 1, sap.LU_UL, sap.Spike),     # one partition: no reduced system
    (12000, 280, 4, 1.0, 0, sap.LU_UL, sap.Block),    # decoupled partitions
    (6600, 1100, 2, 1.0, 1, sap.LU_UL, sap.Spike),    # above the narrow kernels' limit
]


@pytest.mark.parametrize("dtype", ["double", "float"])
@pytest.mark.parametrize("n,K,P,d,dist,fact,ptype", WIDE_CASES)
def test_wide_apply_matches_oracle(n, K, P, d, dist, fact, ptype, dtype):
    band = sap.generate_band_host(n, K, d, dist, seed=n + K)
    A, s, o = setup_pair(band, n, K, P, dtype, fact, ptype)
    assert s.info() == o.info()
    rng = np.random.default_rng(K)
    for _ in range(2):
        v = rng.standard_normal(n)
        z = apply_gpu(s, v)
        zo = o.apply(v)
        assert np.all(np.isfinite(z))
        rel = np.linalg.norm(z - zo) / np.linalg.norm(zo)
        assert rel <= APPLY_TOL[dtype], rel


def test_threshold_override_runs_block_path_on_narrow_band(monkeypatch):
    n, K, P = 30011, 50, 10
    band = sap.generate_band_host(n, K, 1.0, 1, seed=n + K)
    v = np.random.default_rng(1).standard_normal(n)
    _, s_narrow, o = setup_pair(band, n, K, P, "double")
    monkeypatch.setenv("SAPB_WIDE_MIN_K", "32")
    _, s_wide, _ = setup_pair(band, n, K, P, "double")
    zo = o.apply(v)
    for s in (s_narrow, s_wide):
        z = apply_gpu(s, v)
        assert np.linalg.norm(z - zo) / np.linalg.norm(zo) <= 1e-10


def test_wide_fp64_solve_matches_oracle_and_direct():
    n, K, P = 40000, 300, 8
    band = sap.generate_band_host(n, K, 1.0, 1, seed=11)
    xt = np.ones(n)
    b = oracle.spmv_banded(band, n, K, xt)
    A, s, o = setup_pair(band, n, K, P, "double")
    x = np.zeros(n)
    ok = s.solve(sap.MVBanded(A), b, x)
    xo, res = o.solve(b, band=band, K=K, L=2, maxit=100, reltol=1e-10)
    assert ok and res.code == 1
    assert s.getMonitorCode() == 1
    st = s.getStats()
    assert st.relResidualNorm <= 1e-10
    assert abs(st.numIterations - res.iterations) <= 0.5
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9
    xd = sl.solve_banded((K, K), band_to_scipy(band, n, K), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) <= 1e-8


@pytest.mark.parametrize("prec", ["float", "tf32"])
def test_refinement_reaches_fp64_tolerance_with_low_precision_preconditioner(prec):
    # the FP32 / TF32 preconditioner stagnates BiCGStab(2) near FP32
    # accuracy; FP64 refinement sweeps around it reach 1e-10
    from saplibrary_b200.problems import convection_diffusion_csr, csr_matvec
    m, P = 100, 16
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    n = m * m
    A = sap.CsrMatrix(rp, ci, v)
    b = np.random.default_rng(3).standard_normal(n)
    s = sap.Solver(P, sap.Options(dropOffFraction=1e-4, relTol=1e-10, maxNumIterations=100,
                                  refinementSweeps=6), prec=prec)
    s.setup(A)
    assert s.getStats().bandwidth >= 256  # the block path
    x = np.zeros(n)
    assert s.solve(sap.SpmvCusp(A), b, x)
    assert s.getMonitorCode() == 1
    st = s.getStats()
    assert st.relResidualNorm <= 1e-10
    true_rel = np.linalg.norm(b - csr_matvec(rp, ci, v, x)) / np.linalg.norm(b)
    assert true_rel <= 1.01e-10
    assert abs(true_rel - st.relResidualNorm) <= 1e-12


def test_tf32_banded_refinement():
    n, K, P = 40000, 300, 8
    band = sap.generate_band_host(n, K, 1.0, 1, seed=12)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    A = sap.BandedMatrix.from_array(band, n, K)
    opts = sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=sap.LU_UL,
                       relTol=1e-10, maxNumIterations=100, refinementSweeps=4)
    s = sap.Solver(P, opts, prec="tf32")
    s.setup(A)
    x = np.zeros(n)
    assert s.solve(sap.MVBanded(A), b, x)
    assert s.getStats().relResidualNorm <= 1e-10
    assert np.linalg.norm(x - 1.0) / np.sqrt(n) <= 1e-8


@pytest.mark.parametrize("prec", ["double", "tf32", "tf32_f16"])
def test_fgmres_reaches_fp64_tolerance(prec):
    # flexible GMRES keeps the preconditioned directions, so a low-precision
    # preconditioner needs no refinement restarts
    from saplibrary_b200.problems import convection_diffusion_csr, csr_matvec
    m, P = 100, 16
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    n = m * m
    A = sap.CsrMatrix(rp, ci, v)
    b = np.random.default_rng(4).standard_normal(n)
    s = sap.Solver(P, sap.Options(solverType=sap.FGMRES, dropOffFraction=1e-4, relTol=1e-10,
                                  maxNumIterations=200), prec=prec)
    s.setup(A)
    x = np.zeros(n)
    assert s.solve(sap.SpmvCusp(A), b, x)
    assert s.getMonitorCode() == 1
    st = s.getStats()
    assert st.relResidualNorm <= 1e-10
    true_rel = np.linalg.norm(b - csr_matvec(rp, ci, v, x)) / np.linalg.norm(b)
    assert true_rel <= 1.01e-10
    assert abs(true_rel - st.relResidualNorm) <= 1e-12


def test_fgmres_narrow_band_matches_direct():
    n, K, P = 60000, 16, 8
    band = sap.generate_band_host(n, K, 0.9, 2, seed=7)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    A = sap.BandedMatrix.from_array(band, n, K)
    opts = sap.Options(solverType=sap.FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                       factMethod=sap.LU_UL, relTol=1e-10, maxNumIterations=200)
    s = sap.Solver(P, opts, prec="float")
    s.setup(A)
    x = np.zeros(n)
    assert s.solve(sap.MVBanded(A), b, x)
    assert s.getStats().relResidualNorm <= 1e-10
    xd = sl.solve_banded((K, K), band_to_scipy(band, n, K), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) <= 1e-8


def test_cusp_solver_type_is_unsupported():
    n, K = 2000, 4
    band = sap.generate_band_host(n, K, 1.0, 1, seed=2)
    A = sap.BandedMatrix.from_array(band, n, K)
    opts = sap.Options(solverType=sap.CG_C, performReorder=False, variableBandwidth=False, applyScaling=False)
    s = sap.Solver(2, opts, prec="double")
    s.setup(A)
    with pytest.raises(sap.LibraryError):
        s.solve(sap.MVBanded(A), np.ones(n), np.zeros(n))


@pytest.mark.parametrize("dtype", ["double", "float"])
def test_narrow_kernels_forced_on_wide_band(monkeypatch, dtype):
    # bands whose factor window exceeds shared memory go to the block path by
    # default; the narrow kernels (global-memory factor window, chunked
    # sweeps) stay available and correct when forced
    monkeypatch.setenv("SAPB_WIDE_MIN_K", "100000")
    n, K, P = 40000, 170, 8
    band = sap.generate_band_host(n, K, 0.8, 2, seed=n + K)
    A, s, o = setup_pair(band, n, K, P, dtype)
    assert s.blockLayout()[0] == 0  # narrow path
    v = np.random.default_rng(5).standard_normal(n)
    z, zo = apply_gpu(s, v), o.apply(v)
    assert np.linalg.norm(z - zo) / np.linalg.norm(zo) <= APPLY_TOL[dtype]


def test_narrow_var_band_forced(monkeypatch):
    from saplibrary_b200.problems import convection_diffusion_csr
    monkeypatch.setenv("SAPB_WIDE_MIN_K", "100000")
    m, P = 60, 8
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    A = sap.CsrMatrix(rp, ci, v)
    s = sap.Solver(P, sap.Options(dropOffFraction=1e-4, relTol=1e-10), prec="double")
    s.setup(A)
    assert s.blockLayout()[0] == 0 and s.getStats().bandwidth > 108
    o = oracle.SparsePrecond(P, dtype="double", dropFrac=1e-4)
    assert o.setup(rp, ci, v) == 0
    x = np.random.default_rng(6).standard_normal(m * m)
    vd = torch.tensor(x, device="cuda")
    zd = torch.empty_like(vd)
    s.precond(vd, zd)
    zo = o.apply(x)
    assert np.linalg.norm(zd.cpu().numpy() - zo) / np.linalg.norm(zo) <= 1e-10


@pytest.mark.parametrize("n,K,P,fact", [(20000, 300, 4, sap.LU_UL), (24011, 257, 5, sap.LU_only),
                                        (6600, 1100, 2, sap.LU_UL)])
def test_f16_block_storage_apply(n, K, P, fact):
    # the FP16 block-scaled copies change only the storage of the factor
    # blocks read by the sweeps: the apply stays within the FP16 rounding of
    # the same TF32 factors, and both stay near the FP32 oracle's apply
    band = sap.generate_band_host(n, K, 1.0, 1, seed=n + K)
    A = sap.BandedMatrix.from_array(band, n, K)
    s32 = sap.Solver(P, sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=fact),
                     prec="tf32")
    s16 = sap.Solver(P, sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=fact),
                     prec="tf32_f16")
    s32.setup(A)
    s16.setup(A)
    assert s16.blockLayout()[:2] == s32.blockLayout()[:2] and s32.blockLayout()[0] > 0
    assert s16.blockLayout()[2] == 2
    o = oracle.Precond(P, fact=fact, ptype=sap.Spike, dtype="float")
    assert o.setup_banded(band, n, K) == 0
    rng = np.random.default_rng(K)
    for _ in range(2):
        v = rng.standard_normal(n)
        z32, z16, zo = apply_gpu(s32, v), apply_gpu(s16, v), o.apply(v)
        assert np.all(np.isfinite(z16))
        assert np.linalg.norm(z16 - z32) / np.linalg.norm(z32) <= 5e-3
        assert np.linalg.norm(z16 - zo) / np.linalg.norm(zo) <= 3e-2


def test_f16_block_storage_fgmres_banded():
    n, K, P = 40000, 300, 8
    band = sap.generate_band_host(n, K, 1.0, 1, seed=12)
    b = oracle.spmv_banded(band, n, K, np.ones(n))
    A = sap.BandedMatrix.from_array(band, n, K)
    opts = sap.Options(solverType=sap.FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                       factMethod=sap.LU_UL, relTol=1e-10, maxNumIterations=200)
    s = sap.Solver(P, opts, prec="tf32_f16")
    s.setup(A)
    x = np.zeros(n)
    assert s.solve(sap.MVBanded(A), b, x)
    assert s.getStats().relResidualNorm <= 1e-10
    assert np.linalg.norm(x - 1.0) / np.sqrt(n) <= 1e-8


@pytest.mark.parametrize("prec,tol", [("double", 1e-12), ("float", 1e-5), ("tf32_f16", 1e-5)])
def test_persistent_sweep_matches_launch_chain(monkeypatch, prec, tol):
    # the block sweeps as one cooperative launch (group barriers between the
    # block-row steps) against the chain of per-step launches: the same
    # products, summed in slices that may differ
    n, K, P = 24011, 257, 5
    band = sap.generate_band_host(n, K, 0.8, 2, seed=n + K)
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False,
                                  factMethod=sap.LU_only), prec=prec)
    s.setup(A)
    v = np.random.default_rng(5).standard_normal(n)
    monkeypatch.setenv("SAPB_SWEEP_PERSISTENT", "1")
    z1 = apply_gpu(s, v)
    monkeypatch.setenv("SAPB_SWEEP_PERSISTENT", "0")
    z0 = apply_gpu(s, v)
    assert np.all(np.isfinite(z1))
    assert np.linalg.norm(z1 - z0) / np.linalg.norm(z0) <= tol


def test_persistent_sweep_barrier_timeout_is_reported(monkeypatch):
    # a group barrier made to wait for one CTA more than its group has (a
    # count nothing completes): its bounded wait runs out, the kernel
    # returns, the host reports SAP_ERR_DEVICE_TIMEOUT, and the next apply
    # works again
    n, K, P = 24011, 257, 5
    band = sap.generate_band_host(n, K, 0.8, 2, seed=n + K)
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False,
                                  factMethod=sap.LU_only), prec="tf32_f16")
    s.setup(A)
    v = np.random.default_rng(6).standard_normal(n)
    monkeypatch.setenv("SAPB_SWEEP_PERSISTENT", "1")
    z_ok = apply_gpu(s, v)
    monkeypatch.setenv("SAPB_TEST_BARRIER_STALL", "1")
    with pytest.raises(sap.LibraryError) as ei:
        apply_gpu(s, v)
    assert ei.value.code == -104  # SAP_ERR_DEVICE_TIMEOUT
    monkeypatch.delenv("SAPB_TEST_BARRIER_STALL")
    z_again = apply_gpu(s, v)
    assert np.linalg.norm(z_again - z_ok) / np.linalg.norm(z_ok) <= 1e-6
