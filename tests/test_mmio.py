"""Matrix Market input (the reference drivers' cusp::io reader) against
scipy.io.mmread, on the host (no GPU)."""
import numpy as np
import pytest
import scipy.io as sio
import scipy.sparse as sp

import saplibrary_b200 as sap


@pytest.mark.parametrize("symmetry", ["general", "symmetric", "skew-symmetric"])
def test_read_csr_matches_scipy(tmp_path, symmetry):
    rng = np.random.default_rng(1)
    A = sp.random(300, 300, density=0.02, random_state=2, format="coo")
    if symmetry == "symmetric":
        A = (A + A.T).tocoo()
    elif symmetry == "skew-symmetric":
        A = (A - A.T).tocoo()
    path = str(tmp_path / "a.mtx")
    sio.mmwrite(path, A, symmetry=symmetry)
    rp, ci, v, shape = sap.read_matrix_market(path)
    ref = sio.mmread(path).tocsr()
    ref.sum_duplicates()
    ref.sort_indices()
    assert shape == ref.shape
    assert np.array_equal(rp, ref.indptr) and np.array_equal(ci, ref.indices)
    assert np.allclose(v, ref.data, rtol=1e-15, atol=0)


def test_pattern_duplicates_and_vectors(tmp_path):
    path = str(tmp_path / "p.mtx")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n% comment\n3 3 4\n1 1\n2 3\n2 3\n3 2\n")
    rp, ci, v, shape = sap.read_matrix_market(path)
    assert shape == (3, 3)
    assert list(rp) == [0, 1, 2, 3] and list(ci) == [0, 2, 1] and list(v) == [1.0, 2.0, 1.0]
    vec = str(tmp_path / "b.mtx")
    sio.mmwrite(vec, np.arange(5.0).reshape(5, 1))
    assert np.array_equal(sap.read_matrix_market_vector(vec), np.arange(5.0))
    bad = str(tmp_path / "bad.mtx")
    with open(bad, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n")
    with pytest.raises(sap.LibraryError):
        sap.read_matrix_market(bad)
