"""ORACLE — test infrastructure only (not product code).

CPU restatement of the SaP SPIKE-preconditioned BiCGStab(L) solve of the
reference (see sap_oracle.cpp for the per-function citations).  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline / reference leg may use
it, and only as the checker or the CPU baseline; the product library never
loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "sap_oracle.cpp")


SRC2 = os.path.join(HERE, "reorder_oracle.cpp")


def build(force: bool = False) -> str:
    newest = max(os.path.getmtime(SRC), os.path.getmtime(SRC2))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB], check=True)
    return LIB


class OrcResult(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("iterations", ctypes.c_float), ("rhs_norm", ctypes.c_double),
                ("res_norm", ctypes.c_double), ("rel_res_norm", ctypes.c_double), ("n", ctypes.c_int),
                ("K", ctypes.c_int), ("P", ctypes.c_int), ("status", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, ip, dp, i = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
        L.orc_precond_create.restype = vp
        L.orc_precond_create.argtypes = [i, i, i, i, i]
        L.orc_precond_destroy.argtypes = [vp]
        L.orc_setup_banded.argtypes = [vp, i, i, dp]
        L.orc_setup_csr.argtypes = [vp, i, ip, ip, dp]
        L.orc_info.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i)]
        L.orc_apply.argtypes = [vp, dp, dp]
        L.orc_factor_copy.restype = ctypes.c_longlong
        L.orc_factor_copy.argtypes = [vp, i, dp]
        L.orc_spmv_banded.argtypes = [i, i, dp, dp, dp]
        L.orc_spmv_csr.argtypes = [i, ip, ip, dp, dp, dp]
        L.orc_solve.argtypes = [vp, i, i, dp, ip, ip, dp, dp, dp, i, i, ctypes.c_double, ctypes.c_double,
                                ctypes.POINTER(OrcResult)]
        L.orc_num_threads.restype = i
        L.orc_band_lu_sample.restype = ctypes.c_double
        L.orc_band_lu_sample.argtypes = [i, i]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Precond:
    """The oracle's preconditioner: setup on a band or CSR matrix, apply."""

    def __init__(self, P, fact=0, ptype=0, safe=False, dtype="float"):
        self.h = lib().orc_precond_create(int(P), int(fact), int(ptype), int(bool(safe)),
                                          0 if dtype == "float" else 1)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_precond_destroy(self.h)
            self.h = None

    def setup_banded(self, band_rowmajor: np.ndarray, n: int, K: int) -> int:
        self._band = np.ascontiguousarray(band_rowmajor, dtype=np.float64)
        return lib().orc_setup_banded(self.h, n, K, _p(self._band))

    def setup_csr(self, n, rp, ci, v) -> int:
        self._csr = [np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                     np.ascontiguousarray(v, np.float64)]
        return lib().orc_setup_csr(self.h, n, *[_p(a) for a in self._csr])

    def info(self):
        n, K, P = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib().orc_info(self.h, ctypes.byref(n), ctypes.byref(K), ctypes.byref(P))
        return n.value, K.value, P.value

    def apply(self, v: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(v, np.float64)
        z = np.empty_like(v)
        lib().orc_apply(self.h, _p(v), _p(z))
        return z

    def factor(self, which: int) -> np.ndarray:
        """0 band factors, 1 V tips, 2 W tips, 3 LU of S, 4 coupling blocks (as float64)."""
        cnt = lib().orc_factor_copy(self.h, which, None)
        out = np.empty(cnt, np.float64)
        if cnt:
            lib().orc_factor_copy(self.h, which, _p(out))
        return out

    def solve(self, b, x0=None, band=None, K=0, csr=None, L=2, maxit=100, reltol=1e-6, abstol=0.0):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        res = OrcResult()
        if band is not None:
            band = np.ascontiguousarray(band, np.float64)
            lib().orc_solve(self.h, b.size, K, _p(band), None, None, None, _p(b), _p(x), L, maxit, reltol, abstol,
                            ctypes.byref(res))
        else:
            rp, ci, v = [np.ascontiguousarray(a) for a in csr]
            lib().orc_solve(self.h, b.size, 0, None, _p(rp), _p(ci), _p(v), _p(b), _p(x), L, maxit, reltol, abstol,
                            ctypes.byref(res))
        return x, res


def spmv_banded(band, n, K, x):
    band = np.ascontiguousarray(band, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(n)
    lib().orc_spmv_banded(n, K, _p(band), _p(x), _p(y))
    return y


def spmv_csr(rp, ci, v, x):
    rp, ci, v, x = (np.ascontiguousarray(a) for a in (rp, ci, v, x))
    y = np.empty(rp.size - 1)
    lib().orc_spmv_csr(rp.size - 1, _p(rp), _p(ci), _p(v), _p(x), _p(y))
    return y


def band_lu_sample(K: int, steps: int) -> float:
    """Seconds of the first `steps` pivots of the FP64 partition band LU at
    half-bandwidth K (a CPU-baseline timing sample)."""
    return lib().orc_band_lu_sample(int(K), int(steps))


def num_threads() -> int:
    return lib().orc_num_threads()


class SparseInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("nnz", ctypes.c_int), ("K", ctypes.c_int), ("P", ctypes.c_int),
                ("k_db", ctypes.c_int), ("k_reorder", ctypes.c_int), ("varBand", ctypes.c_int),
                ("status", ctypes.c_int), ("drop_actual", ctypes.c_double)]


_sparse_sigs = False


def _sparse_lib():
    global _sparse_sigs
    L = lib()
    if not _sparse_sigs:
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_sparse_create.restype = vp
        L.orc_sparse_create.argtypes = [i, i, i, i, d, i, i, i]
        L.orc_sparse_destroy.argtypes = [vp]
        L.orc_sparse_setup.argtypes = [vp, i, vp, vp, vp, i, ctypes.c_char_p, i]
        L.orc_sparse_info_get.argtypes = [vp, ctypes.POINTER(SparseInfo)]
        L.orc_sparse_ints.restype = ctypes.c_longlong
        L.orc_sparse_ints.argtypes = [vp, i, vp]
        L.orc_sparse_reals.restype = ctypes.c_longlong
        L.orc_sparse_reals.argtypes = [vp, i, vp]
        L.orc_sparse_apply.argtypes = [vp, vp, vp]
        L.orc_sparse_solve.argtypes = [vp, i, vp, vp, vp, vp, vp, i, i, d, d, ctypes.POINTER(OrcResult)]
        _sparse_sigs = True
    return L


INT_NAMES = ["dbRowPerm", "optReordering", "optPerm", "secondReorder", "secondPerm", "first_rows", "ks",
             "finalPerm", "finalReordering", "offDiagWidths_left", "offDiagWidths_right", "offDiagPerms_left",
             "offDiagPerms_right", "ks_col", "ks_row"]


class SparsePrecond:
    """The oracle's sparse setup: DB + RCM + drop-off + (variable) band
    assembly of sap/graph.h, then the variable-band SPIKE preconditioner."""

    def __init__(self, P, dtype="float", doDB=True, scale=True, dropFrac=0.0, maxBandwidth=2**31 - 1,
                 varBand=True, safe=False):
        self.h = _sparse_lib().orc_sparse_create(int(P), 0 if dtype == "float" else 1, int(doDB), int(scale),
                                                 float(dropFrac), int(maxBandwidth), int(varBand), int(safe))

    def __del__(self):
        if getattr(self, "h", None):
            _sparse_lib().orc_sparse_destroy(self.h)
            self.h = None

    def setup(self, rp, ci, v, factor=True, band=True):
        """factor: also factor the band; band=False (with factor=False) stops
        after the permutations, without assembling the band storage."""
        self._csr = [np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                     np.ascontiguousarray(v, np.float64)]
        msg = ctypes.create_string_buffer(256)
        mode = 1 if factor else (0 if band else 2)
        rc = _sparse_lib().orc_sparse_setup(self.h, self._csr[0].size - 1, *[_p(a) for a in self._csr],
                                            mode, msg, 256)
        self.message = msg.value.decode()
        return rc

    def info(self) -> SparseInfo:
        s = SparseInfo()
        _sparse_lib().orc_sparse_info_get(self.h, ctypes.byref(s))
        return s

    def ints(self, name: str) -> np.ndarray:
        w = INT_NAMES.index(name)
        cnt = _sparse_lib().orc_sparse_ints(self.h, w, None)
        out = np.empty(cnt, np.int32)
        if cnt:
            _sparse_lib().orc_sparse_ints(self.h, w, _p(out))
        return out

    def reals(self, which: int) -> np.ndarray:
        cnt = _sparse_lib().orc_sparse_reals(self.h, which, None)
        out = np.empty(cnt, np.float64)
        if cnt:
            _sparse_lib().orc_sparse_reals(self.h, which, _p(out))
        return out

    def apply(self, v):
        v = np.ascontiguousarray(v, np.float64)
        z = np.empty_like(v)
        _sparse_lib().orc_sparse_apply(self.h, _p(v), _p(z))
        return z

    def solve(self, b, x0=None, L=2, maxit=100, reltol=1e-6, abstol=0.0):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        res = OrcResult()
        rp, ci, v = self._csr
        _sparse_lib().orc_sparse_solve(self.h, b.size, _p(rp), _p(ci), _p(v), _p(b), _p(x), L, maxit, reltol,
                                       abstol, ctypes.byref(res))
        return x, res


# ---- the reference's own reordering pipeline (sap/graph.h) -----------------------
# oracle/_ref/libref_graph.so is sap/graph.h of the reference compiled from its
# source tree against the CUSP stand-in in oracle/ref_graph (build_ref.sh);
# it needs a GPU at run time (DB's device vectors and weight kernel).
REF_LIB = os.path.join(HERE, "_ref", "libref_graph.so")
REF_SRC = "/root/reference"


def build_ref(force: bool = False) -> str | None:
    """Compile the reference's graph.h when the reference tree is present
    (this container); on a machine without it the prebuilt library is used."""
    if not os.path.isdir(REF_SRC):
        return REF_LIB if os.path.exists(REF_LIB) else None
    srcs = [os.path.join(HERE, "ref_graph", "ref_graph_driver.cu"), os.path.join(HERE, "ref_graph", "cusp", "shim.h")]
    newest = max(os.path.getmtime(s) for s in srcs)
    if force or not os.path.exists(REF_LIB) or os.path.getmtime(REF_LIB) < newest:
        subprocess.run(["sh", os.path.join(HERE, "ref_graph", "build_ref.sh"), REF_SRC], check=True)
    return REF_LIB


class RefInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("K", ctypes.c_int), ("P", ctypes.c_int), ("k_db", ctypes.c_int),
                ("k_reorder", ctypes.c_int), ("varBand", ctypes.c_int), ("status", ctypes.c_int),
                ("drop_actual", ctypes.c_double)]


_ref = None


def ref_lib():
    """The reference's graph.h pipeline (None when its library is absent)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        L = ctypes.CDLL(REF_LIB)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ref_graph_run.restype = vp
        L.ref_graph_run.argtypes = [i, vp, vp, vp, i, i, d, i, i, i, i, ctypes.c_char_p, i]
        L.ref_graph_info_get.argtypes = [vp, ctypes.POINTER(RefInfo)]
        L.ref_graph_ints.restype = ctypes.c_longlong
        L.ref_graph_ints.argtypes = [vp, i, vp]
        L.ref_graph_destroy.argtypes = [vp]
        _ref = L
    return _ref


class RefGraph:
    """One run of the reference's reorder pipeline (Graph::reorder, dropOff,
    assembleOffDiagMatrices, secondLevelReordering, assembleBandedMatrix and
    the permutation composition of Precond::transformToBandedMatrix) on a
    CSR matrix; the integer outputs use the names of INT_NAMES."""

    def __init__(self, rp, ci, v, P, dtype="float", doDB=True, scale=True, dropFrac=0.0, maxBandwidth=2**31 - 1,
                 varBand=True):
        L = ref_lib()
        if L is None:
            raise RuntimeError("oracle/_ref/libref_graph.so is not built")
        self._csr = [np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                     np.ascontiguousarray(v, np.float64)]
        msg = ctypes.create_string_buffer(256)
        self.h = L.ref_graph_run(self._csr[0].size - 1, *[_p(a) for a in self._csr], 0 if dtype == "float" else 1,
                                 int(P), float(dropFrac), int(doDB), int(scale), int(maxBandwidth), int(varBand),
                                 msg, 256)
        self.message = msg.value.decode()

    def __del__(self):
        if getattr(self, "h", None):
            ref_lib().ref_graph_destroy(self.h)
            self.h = None

    def info(self) -> RefInfo:
        s = RefInfo()
        ref_lib().ref_graph_info_get(self.h, ctypes.byref(s))
        return s

    def ints(self, name: str) -> np.ndarray:
        w = INT_NAMES.index(name)
        cnt = ref_lib().ref_graph_ints(self.h, w, None)
        out = np.empty(cnt, np.int32)
        if cnt:
            ref_lib().ref_graph_ints(self.h, w, _p(out))
        return out
