"""Diagonal scaling of the TF32 forms (banded and unreordered CSR setups):
the band is scaled to S A S with power-of-two S chosen from the diagonal
(s_r^2 |a_rr| in [0.5, 2)) before the TF32 factorisation, and the apply
scales its input and output by S.  Powers of two scale without rounding, so a
matrix and right-hand side multiplied by 2^-40 -- every pivot far below the
reference's 1e-7 boost / zero-pivot threshold -- give the TF32 form exactly
the solution of the unscaled system, bit for bit, while the FP32 form (the
reference's PrecValueType, unscaled) reports the zero pivots as the
reference does.  Covers the narrow (K = 40) and wide (K = 300) paths."""
import numpy as np
import pytest

import saplibrary_b200 as sap

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _opts():
    return sap.Options(solverType=sap.FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                       factMethod=sap.LU_UL, relTol=1e-10, maxNumIterations=200)


def _solve(band, n, K, P, b, prec):
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, _opts(), prec=prec)
    s.setup(A)
    x = np.zeros(n)
    ok = s.solve(sap.MVBanded(A), b, x)
    return ok, x, s.getStats()


@pytest.mark.parametrize("n,K,P", [(60000, 40, 8), (40000, 300, 8)])
def test_tf32_form_is_invariant_under_power_of_two_scaling(n, K, P):
    band = sap.generate_band_host(n, K, 0.9, 2, seed=K)
    b = np.random.default_rng(K).standard_normal(n)
    ok1, x1, st1 = _solve(band, n, K, P, b, "tf32")
    f = 2.0 ** -40
    ok2, x2, st2 = _solve(band * f, n, K, P, b * f, "tf32")
    assert ok1 and ok2
    assert st1.relResidualNorm <= 1e-10 and st2.relResidualNorm <= 1e-10
    assert st1.numIterations == st2.numIterations
    assert np.array_equal(x1, x2)


def test_fp32_form_keeps_the_reference_thresholds():
    n, K, P = 60000, 40, 8
    band = sap.generate_band_host(n, K, 0.9, 2, seed=3) * 2.0 ** -40
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, _opts(), prec="float")
    with pytest.raises(sap.SystemError) as e:
        s.setup(A)
    assert e.value.reason == sap.SystemError.Zero_pivoting
