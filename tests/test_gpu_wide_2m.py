"""The mixed-precision wide-band workload at its full size: N = 2,000,000,
half-bandwidth K = 200, off-diagonals N(0, 1), diagonal 0.8 times the row's
off-diagonal magnitude sum, P = 32, coupled SPIKE with LU_UL on a constant
band (the reference's banded preset, examples/synthetic_banded/
driver_banded.cu:166-170), solved to the FP64 relative residual 1e-10 of
sap/monitor.h:291-314 from x = 0.

Every precision form (FP64 preconditioner with BiCGStab(2), TF32 and FP32
preconditioners with flexible GMRES) must converge with the monitor's code
1, a true FP64 residual within the criterion, and an error against the
known solution at FP64 level; the iteration count of each form is printed.
The error against an FP64 direct banded LU with partial pivoting (LAPACK
gbsv through scipy) is checked on the same family at a tenth of the size."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle
import saplibrary_b200 as sap
from tests.helpers import band_to_scipy

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORMS = [("double", sap.BiCGStab2), ("tf32", sap.FGMRES), ("float", sap.FGMRES)]


def _opts(solver):
    return sap.Options(solverType=solver, performReorder=False, variableBandwidth=False, applyScaling=False,
                       factMethod=sap.LU_UL, relTol=1e-10, maxNumIterations=400)


def test_2m_k200_every_precision_form_reaches_fp64_tolerance():
    n, K, P = 2_000_000, 200, 32
    A = sap.BandedMatrix(n, K, 0.8, dist=2, seed=1)
    spmv = sap.MVBanded(A)
    x_true = torch.tensor(np.random.default_rng(5).standard_normal(n), device="cuda")
    b = torch.empty_like(x_true)
    spmv(x_true, b)
    iters = {}
    for prec, solver in FORMS:
        s = sap.Solver(P, _opts(solver), prec=prec)
        s.setup(A)
        assert s.info() == (n, K, P)
        x = torch.zeros_like(b)
        assert s.solve(spmv, b, x), prec
        assert s.getMonitorCode() == 1 and s.getMonitorMessage() == "Converged"
        r = torch.empty_like(b)
        spmv(x, r)
        true_rel = float(torch.linalg.norm(b - r) / torch.linalg.norm(b))
        assert true_rel <= 1.01e-10, (prec, true_rel)
        err = float(torch.linalg.norm(x - x_true) / torch.linalg.norm(x_true))
        assert err <= 1e-9, (prec, err)
        iters[prec] = (s.getStats().numIterations, err)
        del s
        torch.cuda.empty_cache()
    print("iterations and error vs the known solution per precision:", iters)


def test_k200_family_matches_fp64_direct_banded_lu():
    n, K, P = 200_000, 200, 32
    band = sap.generate_band_host(n, K, 0.8, 2, seed=2)
    A = sap.BandedMatrix.from_array(band, n, K)
    b = oracle.spmv_banded(band, n, K, np.random.default_rng(6).standard_normal(n))
    xd = sl.solve_banded((K, K), band_to_scipy(band, n, K), b)
    for prec, solver in FORMS:
        s = sap.Solver(P, _opts(solver), prec=prec)
        s.setup(A)
        x = np.zeros(n)
        assert s.solve(sap.MVBanded(A), b, x), prec
        assert s.getStats().relResidualNorm <= 1e-10
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) <= 1e-9, prec
