"""Batched solve of independent banded systems (sap_batch_banded_solve):
every system meets its own relative-residual criterion, checked here with
an independent FP64 matvec, and the solutions match direct banded solves."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle
import saplibrary_b200 as sap
from saplibrary_b200 import ensemble
from tests.helpers import band_to_scipy

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("prec", ["float", "double"])
def test_batch_meets_per_system_tolerance(prec):
    bands, ks, bs = ensemble.make_ensemble(40, seed=5, n_min=2000, n_max=20000, ks=(8, 16, 32, 64))
    xs, res, sec = sap.solve_batch(bands, ks, bs, 4, ensemble.options(1e-10), prec)
    assert sec > 0
    for band, K, b, x, r in zip(bands, ks, bs, xs, res):
        n = len(b)
        true = np.linalg.norm(b - oracle.spmv_banded(band, n, K, x)) / np.linalg.norm(b)
        assert r[2] and r[0] <= 1e-10 and true <= 1.05e-10, (n, K, r, true)
        assert abs(true - r[0]) <= 1e-12
    for i in (0, 7, 21):
        n, K = len(bs[i]), ks[i]
        xd = sl.solve_banded((K, K), band_to_scipy(bands[i], n, K), bs[i])
        assert np.linalg.norm(xs[i] - xd) / np.linalg.norm(xd) <= 1e-8


def test_batch_rejects_bad_input():
    band = sap.generate_band_host(100, 4, 1.0, 1, seed=1)
    with pytest.raises(sap.LibraryError):
        sap.solve_batch([band], [200], [np.ones(100)], 2, ensemble.options(), "float")
