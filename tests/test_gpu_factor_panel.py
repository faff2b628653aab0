"""The panel-blocked narrow-band factorisation (k_factor_panel: one warp
factors NB = 8 pivots in registers with reciprocal-based exact quotients,
then all warps apply them to the next K columns; the U entries divided by
their pivots in a separate pass, k_factor_postdiv) against the
one-pivot-at-a-time ring kernel it replaces (k_factor_smem, selected with
SAPB_FACTOR_KERNEL=ring).  Both apply the same updates to every element in
the same order with the same rounding, so the factors, and hence every
preconditioner apply, are equal bit for bit.  Shapes cover K below the panel
width, partitions shorter than a panel, ragged last panels, LU_only and LU_UL
(mirrored UL jobs), pivot boosting, both precisions, the variable-band sparse
path, and, through the oracle, the tolerance of the existing apply tests."""
import os

import numpy as np
import pytest

import oracle
import saplibrary_b200 as sap
from saplibrary_b200.problems import convection_diffusion_csr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = [  # n, K, P, d, dist, fact, safe
    (20000, 10, 4, 1.0, 1, sap.LU_UL, False),
    (30011, 50, 10, 1.0, 1, sap.LU_UL, False),
    (15000, 33, 5, 1.0, 0, sap.LU_only, False),
    (9000, 75, 4, 1.0, 1, sap.LU_UL, False),
    (9001, 100, 6, 1.0, 1, sap.LU_UL, False),
    (12000, 8, 6, 0.8, 2, sap.LU_UL, True),   # boosted pivots
    (5003, 1, 3, 1.0, 1, sap.LU_UL, False),
    (4001, 3, 5, 1.0, 1, sap.LU_only, False),
    (2000, 7, 4, 1.0, 1, sap.LU_UL, False),
    (300, 30, 8, 1.0, 1, sap.LU_UL, False),   # partitions of ~37 rows
    (70, 9, 7, 1.0, 1, sap.LU_UL, False),     # partitions of 10 rows
    (5000, 20, 1, 1.0, 1, sap.LU_UL, False),
]


def _opts(fact, safe):
    return sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=fact,
                       safeFactorization=safe, precondType=sap.Spike)


def _apply(s, v):
    vd = torch.tensor(v, device="cuda", dtype=torch.float64)
    zd = torch.empty_like(vd)
    s.precond(vd, zd)
    return zd.cpu().numpy()


def _with_kernel(kernel, make):
    old = os.environ.pop("SAPB_FACTOR_KERNEL", None)
    if kernel:
        os.environ["SAPB_FACTOR_KERNEL"] = kernel
    try:
        return make()
    finally:
        os.environ.pop("SAPB_FACTOR_KERNEL", None)
        if old is not None:
            os.environ["SAPB_FACTOR_KERNEL"] = old


@pytest.mark.parametrize("dtype", ["double", "float"])
@pytest.mark.parametrize("n,K,P,d,dist,fact,safe", CASES)
def test_panel_factor_equals_ring_factor_bitwise(n, K, P, d, dist, fact, safe, dtype):
    band = sap.generate_band_host(n, K, d, dist, seed=n + K)
    A = sap.BandedMatrix.from_array(band, n, K)
    v = np.random.default_rng(K + 1).standard_normal(n)

    def solve_apply():
        s = sap.Solver(P, _opts(fact, safe), prec=dtype)
        s.setup(A)
        return _apply(s, v)

    z_ring = _with_kernel("ring", solve_apply)
    z = _with_kernel(None, solve_apply)
    assert np.all(np.isfinite(z))
    assert np.array_equal(z_ring, z)


@pytest.mark.parametrize("dtype", ["double", "float"])
def test_panel_factor_variable_band_sparse_path(dtype):
    rp, ci, v, _ = convection_diffusion_csr(m=60, fill_reach=300, seed=7)
    n = rp.size - 1
    x = np.random.default_rng(3).standard_normal(n)

    def solve_apply():
        s = sap.Solver(8, sap.Options(dropOffFraction=1e-3), prec=dtype)
        s.setup(sap.CsrMatrix(rp, ci, v))
        return _apply(s, x)

    assert np.array_equal(_with_kernel("ring", solve_apply), _with_kernel(None, solve_apply))


def test_panel_factor_matches_oracle_at_config0_shape():
    n, K, P = 200000, 50, 10
    band = sap.generate_band_host(n, K, 1.0, 1, seed=11)
    A = sap.BandedMatrix.from_array(band, n, K)
    s = sap.Solver(P, _opts(sap.LU_UL, False), prec="double")
    s.setup(A)
    o = oracle.Precond(P, fact=sap.LU_UL, ptype=sap.Spike, safe=False, dtype="double")
    assert o.setup_banded(band, n, K) == 0
    v = np.random.default_rng(5).standard_normal(n)
    z, zo = _apply(s, v), o.apply(v)
    assert np.linalg.norm(z - zo) / np.linalg.norm(zo) <= 1e-10
