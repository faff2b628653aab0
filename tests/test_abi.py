"""The C ABI library: loads without a GPU, exports every symbol declared in
include/sap_b200.h, host-side logic (options defaults, generator)."""
import ctypes
import os
import re

import numpy as np

import saplibrary_b200 as sap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "sap_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(sap_[a-z0-9_]+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(os.path.join(ROOT, "saplibrary_b200", "libsap_b200.so"))
    names = declared_symbols()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    assert set(sap.EXPORTED_SYMBOLS) <= set(names)


def test_options_defaults_match_reference():
    # Options::Options() (sap/solver.h:233-256)
    c = sap._COptions()
    assert sap._lib.sap_options_default(ctypes.byref(c)) == 0
    py = sap.Options()
    for name, _ in sap._COptions._fields_:
        assert getattr(c, name) == getattr(py, name), name
    assert c.solverType == sap.BiCGStab2 and c.maxNumIterations == 100 and c.relTol == 1e-6
    assert c.factMethod == sap.LU_only and c.variableBandwidth == 1 and c.ilu_level == -1


def test_generator_is_deterministic_and_dominant():
    for dist in (0, 1, 2):
        a = sap.generate_band_host(500, 6, 1.0, dist, seed=9)
        b = sap.generate_band_host(500, 6, 1.0, dist, seed=9)
        assert np.array_equal(a, b)
        A = a.reshape(500, 13)
        diag = A[:, 6]
        off = np.abs(A).sum(1) - np.abs(diag)
        assert np.allclose(diag, off)  # d = 1: diag = sum |off-diagonals|
        # out-of-range band positions stay zero
        assert np.all(A[0, :6] == 0) and np.all(A[-1, 7:] == 0)
    u = sap.generate_band_host(2000, 4, 1.0, 1, seed=1).reshape(2000, 9)
    offd = np.delete(u, 4, axis=1)
    assert offd.min() >= -1.0 and offd.max() <= 1.0
    c = sap.generate_band_host(2000, 4, 1.0, 1, seed=2)
    assert not np.array_equal(u.ravel(), c)


def test_invalid_arguments_are_rejected_without_gpu():
    out = np.zeros(10)
    rc = sap._lib.sap_generate_band_host(5, 7, 1.0, 1, 0, ctypes.c_void_p(out.ctypes.data))
    assert rc == -100  # SAP_ERR_INVALID_ARGUMENT: k >= n
    assert b"invalid" in sap._lib.sap_last_error()
