"""Solver::update (sap/solver.h:421-462, sap/precond.h:751-900) on the GPU.

update(entries) keeps the setup's permutations, partitions and DB scale
factors and refreshes the values: entries (input CSR order) times the scale
factor of their position, scattered into the band and the coupling blocks,
then the factorisation, spike tips and reduced system are recomputed.
Checks: an update with the setup's own values reproduces the setup's
preconditioner bit-exactly; on the path without reordering an update equals
a fresh setup of the new matrix bit-exactly; updated solvers solve the new
system to the FP64 tolerance.
"""
import numpy as np
import pytest

import saplibrary_b200 as sap
from saplibrary_b200.problems import convection_diffusion_csr, csr_matvec
from tests.helpers import band_to_csr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def apply(s, v):
    vd = torch.tensor(v, device="cuda")
    zd = torch.empty_like(vd)
    s.precond(vd, zd)
    return zd.cpu().numpy()


def perturbed(v, seed):
    return v * np.random.default_rng(seed).uniform(0.9, 1.1, v.size)


@pytest.mark.parametrize("m,P,prec", [(30, 4, "double"), (60, 8, "double"), (60, 8, "tf32")])
def test_sparse_update_reproduces_setup_and_solves_new_matrix(m, P, prec):
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    n = m * m
    opts = sap.Options(dropOffFraction=1e-4, relTol=1e-10, maxNumIterations=200, trackReordering=True,
                       solverType=sap.FGMRES if prec == "tf32" else sap.BiCGStab2)
    s = sap.Solver(P, opts, prec=prec)
    A = sap.CsrMatrix(rp, ci, v)
    s.setup(A)
    x0 = np.random.default_rng(1).standard_normal(n)
    z_setup = apply(s, x0)
    # update with the setup's own values: the same preconditioner
    assert s.update(v.copy())
    assert np.array_equal(apply(s, x0), z_setup)
    # new values on the same pattern: the new system solves to 1e-10
    v2 = perturbed(v, 2)
    assert s.update(v2)
    assert s.getStats().timeUpdate > 0
    A2 = sap.CsrMatrix(rp, ci, v2)
    b = np.random.default_rng(3).standard_normal(n)
    x = np.zeros(n)
    assert s.solve(sap.SpmvCusp(A2), b, x)
    assert s.getMonitorCode() == 1
    assert np.linalg.norm(b - csr_matvec(rp, ci, v2, x)) / np.linalg.norm(b) <= 1.01e-10
    # back to the original values: the original preconditioner again
    assert s.update(v.copy())
    assert np.array_equal(apply(s, x0), z_setup)


@pytest.mark.parametrize("prec", ["double", "float"])
def test_update_without_reordering_equals_fresh_setup(prec):
    n, K, P = 20000, 12, 5
    band = sap.generate_band_host(n, K, 1.0, 1, seed=9)
    rp, ci, v = band_to_csr(band, n, K)
    v2 = perturbed(v, 4)
    opts = sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=sap.LU_UL,
                       trackReordering=True, relTol=1e-10)
    s = sap.Solver(P, opts, prec=prec)
    s.setup(sap.CsrMatrix(rp, ci, v))
    assert s.update(v2)
    fresh = sap.Solver(P, opts, prec=prec)
    fresh.setup(sap.CsrMatrix(rp, ci, v2))
    x0 = np.random.default_rng(5).standard_normal(n)
    assert np.array_equal(apply(s, x0), apply(fresh, x0))


def test_update_constant_band_after_reordering():
    m, P = 40, 4
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    opts = sap.Options(dropOffFraction=1e-4, variableBandwidth=False, trackReordering=True, relTol=1e-10)
    s = sap.Solver(P, opts, prec="double")
    s.setup(sap.CsrMatrix(rp, ci, v))
    x0 = np.random.default_rng(6).standard_normal(m * m)
    z = apply(s, x0)
    assert s.update(perturbed(v, 7))
    assert s.update(v.copy())
    assert np.array_equal(apply(s, x0), z)


def test_update_pattern_change_and_illegal_calls():
    m, P = 30, 4
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    s = sap.Solver(P, sap.Options(trackReordering=True), prec="double")
    with pytest.raises(sap.SystemError) as e:
        s.update(v.copy())
    assert e.value.reason == sap.SystemError.Illegal_update
    s.setup(sap.CsrMatrix(rp, ci, v))
    assert not s.update(np.ones(v.size + 1))  # nnz changed: rejected (solver.h:434-435)
    s2 = sap.Solver(P, sap.Options(trackReordering=False), prec="double")
    s2.setup(sap.CsrMatrix(rp, ci, v))
    with pytest.raises(sap.SystemError) as e:
        s2.update(v.copy())
    assert e.value.reason == sap.SystemError.Illegal_update
    # a BandedMatrix setup has no entry maps
    n, K = 2000, 4
    band = sap.generate_band_host(n, K, 1.0, 1, seed=2)
    s3 = sap.Solver(2, sap.Options(performReorder=False, variableBandwidth=False, trackReordering=True),
                    prec="double")
    s3.setup(sap.BandedMatrix.from_array(band, n, K))
    with pytest.raises(sap.LibraryError):
        s3.update(np.ones(n * (2 * K + 1)))
