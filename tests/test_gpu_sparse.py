"""The reordered sparse path on the GPU against the oracle: DB, RCM,
drop-off, second-level RCM and the variable band bit-exact; the
preconditioner apply and the FP64 solve at the stated tolerances."""
import numpy as np
import pytest

import oracle
import saplibrary_b200 as sap
from saplibrary_b200.problems import convection_diffusion_csr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = [(30, 4), (60, 8), (100, 16)]


def setup_pair(m, P, dtype, drop=1e-4):
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    A = sap.CsrMatrix(rp, ci, v)
    s = sap.Solver(P, sap.Options(dropOffFraction=drop, relTol=1e-10, maxNumIterations=100), prec=dtype)
    s.setup(A)
    o = oracle.SparsePrecond(P, dtype=dtype, dropFrac=drop)
    assert o.setup(rp, ci, v) == 0
    return (rp, ci, v), A, s, o


@pytest.mark.parametrize("dtype", ["double", "float"])
@pytest.mark.parametrize("m,P", CASES)
def test_reordering_is_bit_exact(m, P, dtype):
    _, A, s, o = setup_pair(m, P, dtype)
    inf, st = o.info(), s.getStats()
    assert (st.bandwidthDB, st.bandwidthReorder, st.bandwidth, st.numPartitions) == \
        (inf.k_db, inf.k_reorder, inf.K, inf.P)
    assert st.actualDropOff == inf.drop_actual
    for name in ("dbRowPerm", "finalPerm", "finalReordering", "first_rows", "ks"):
        assert np.array_equal(s.getReorder(name), o.ints(name)), name


@pytest.mark.parametrize("dtype", ["double", "float"])
@pytest.mark.parametrize("m,P", CASES)
def test_sparse_apply_matches_oracle(m, P, dtype):
    _, A, s, o = setup_pair(m, P, dtype)
    n = m * m
    rng = np.random.default_rng(m)
    for _ in range(2):
        v = rng.standard_normal(n)
        vd = torch.tensor(v, device="cuda")
        zd = torch.empty_like(vd)
        s.precond(vd, zd)
        zo = o.apply(v)
        rel = np.linalg.norm(zd.cpu().numpy() - zo) / np.linalg.norm(zo)
        assert rel <= (1e-10 if dtype == "double" else 2e-4), rel


@pytest.mark.parametrize("m,P", CASES)
def test_sparse_fp64_solve_matches_oracle(m, P):
    (rp, ci, v), A, s, o = setup_pair(m, P, "double")
    n = m * m
    b = np.random.default_rng(7).standard_normal(n)
    x = np.zeros(n)
    ok = s.solve(sap.SpmvCusp(A), b, x)
    xo, res = o.solve(b, maxit=100, reltol=1e-10)
    assert ok and res.code == 1 and s.getMonitorCode() == 1
    assert s.getStats().numIterations == res.iterations
    assert s.getStats().relResidualNorm <= 1e-10
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-8


@pytest.mark.parametrize("dtype", ["double", "float"])
def test_config1_size_permutations_bit_exact(dtype):
    # the 1M-row reordered sparse workload: DB, RCM, drop-off and the
    # second-level reordering against the oracle at full size (permutations
    # only: the oracle does not assemble the band)
    m, P = 1000, 16
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=1)
    o = oracle.SparsePrecond(P, dtype=dtype, dropFrac=1e-4)
    assert o.setup(rp, ci, v, factor=False, band=False) == 0
    A = sap.CsrMatrix(rp, ci, v)
    s = sap.Solver(P, sap.Options(dropOffFraction=1e-4, relTol=1e-10), prec="tf32" if dtype == "float" else dtype)
    s.setup(A)
    inf, st = o.info(), s.getStats()
    assert (st.bandwidthDB, st.bandwidthReorder, st.bandwidth, st.numPartitions) == \
        (inf.k_db, inf.k_reorder, inf.K, inf.P)
    assert st.actualDropOff == inf.drop_actual
    for name in ("dbRowPerm", "finalPerm", "finalReordering", "first_rows", "ks"):
        assert np.array_equal(s.getReorder(name), o.ints(name)), name
