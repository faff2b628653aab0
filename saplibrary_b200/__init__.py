"""saplibrary_b200 — B200-native SPIKE-preconditioned Krylov solver.

Python mirror of the reference's public surface (spikegpu/SaPLibrary):
``Options`` (sap/solver.h:52-81), ``Stats`` (sap/solver.h:89-140),
``Solver`` (sap/solver.h:153-225), ``BandedMatrix`` (sap/banded_matrix.h),
``MVBanded`` / ``SpmvCusp`` (sap/spmv.h) and ``SystemError``
(sap/exception.h).  Every call goes through the C ABI of libsap_b200.so
(include/sap_b200.h); there is no CPU fallback: importing the package fails
when the shared library is missing.

Arrays: numpy float64 arrays are host buffers; torch CUDA tensors (float64)
are device buffers and are passed by pointer without copies.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsap_b200.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"saplibrary_b200: {_LIB_PATH} is missing; build it with `python saplibrary_b200/build.py`")
_lib = ctypes.CDLL(_LIB_PATH)

# ---- enums (sap/common.h) ----------------------------------------------------
BiCGStab_C, GMRES_C, CG_C, CR_C, BiCGStab1, BiCGStab2, BiCGStab, MINRES = range(8)
# extension: flexible GMRES(50) with FP64 Arnoldi (tolerates FP32 / TF32 preconditioners)
FGMRES = 8
LU_UL, LU_only = 0, 1
Spike, Block, NoPrecond = 0, 1, 2
HOST, DEVICE = 0, 1


class SystemError(RuntimeError):  # noqa: A001 - mirrors sap::system_error
    """sap::system_error (sap/exception.h:13-45); `reason` is the Reason code."""
    Zero_pivoting = -1
    Negative_DB_weight = -2
    Illegal_update = -3
    Illegal_solve = -4
    Matrix_singular = -5

    def __init__(self, reason: int, what: str):
        super().__init__(what)
        self.reason = reason


class LibraryError(RuntimeError):
    """A failure with no reference counterpart (CUDA error, bad argument...)."""

    def __init__(self, code: int, what: str):
        super().__init__(f"[{code}] {what}")
        self.code = code


class _COptions(ctypes.Structure):
    _fields_ = [("solverType", ctypes.c_int), ("maxNumIterations", ctypes.c_int), ("relTol", ctypes.c_double),
                ("absTol", ctypes.c_double), ("testDB", ctypes.c_int), ("isSPD", ctypes.c_int),
                ("saveMem", ctypes.c_int), ("performReorder", ctypes.c_int), ("performDB", ctypes.c_int),
                ("dbFirstStageOnly", ctypes.c_int), ("applyScaling", ctypes.c_int), ("maxBandwidth", ctypes.c_int),
                ("gpuCount", ctypes.c_int), ("dropOffFraction", ctypes.c_double), ("factMethod", ctypes.c_int),
                ("precondType", ctypes.c_int), ("safeFactorization", ctypes.c_int),
                ("variableBandwidth", ctypes.c_int), ("trackReordering", ctypes.c_int), ("useBCR", ctypes.c_int),
                ("ilu_level", ctypes.c_int), ("refinementSweeps", ctypes.c_int)]


_STAT_FIELDS = (["timeSetup", "timeUpdate", "timeSolve", "time_DB", "time_DB_pre", "time_DB_first",
                 "time_DB_second", "time_DB_post", "d_p1", "d_p1_ori", "diag_dom", "diag_dom_ori",
                 "time_reorder", "time_dropOff", "time_cpu_assemble", "time_transfer", "time_toBanded",
                 "time_offDiags", "time_bandLU", "time_bandUL", "time_fullLU", "time_assembly", "time_shuffle"],
                ["bandwidthReorder", "bandwidthDB", "bandwidth"], ["nuKf", "flops_LU"], ["numPartitions"],
                ["actualDropOff"], ["numIterations"], ["rhsNorm", "residualNorm", "relResidualNorm"],
                ["actual_nnz"])
_STAT_TYPES = (ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_float,
               ctypes.c_double, ctypes.c_int)


class _CStats(ctypes.Structure):
    _fields_ = [(name, t) for group, t in zip(_STAT_FIELDS, _STAT_TYPES) for name in group]


_vp, _i, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_pp = ctypes.POINTER(ctypes.c_void_p)
_sig = {
    "sap_last_error": (ctypes.c_char_p, []),
    "sap_kernel_launch_count": (ctypes.c_int64, []),
    "sap_library_call_count": (ctypes.c_int64, []),
    "sap_mm_read_csr": (_i, [ctypes.c_char_p, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_int64),
                             _vp, _vp, _vp]),
    "sap_mm_read_vector": (_i, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64), _vp]),
    "sap_mm_last_error": (ctypes.c_char_p, []),
    "sap_batch_banded_solve": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _i, ctypes.c_void_p, _i, _vp,
                                    ctypes.POINTER(ctypes.c_double)]),
    "sap_mlp_create": (_i, [_i, _i, _i, _i, ctypes.c_uint64, _pp]),
    "sap_mlp_destroy": (_i, [_vp]),
    "sap_mlp_num_params": (_i, [_vp]),
    "sap_mlp_get_params": (_i, [_vp, _vp]),
    "sap_mlp_set_params": (_i, [_vp, _vp]),
    "sap_mlp_forward": (_i, [_vp, _vp, _i, _vp]),
    "sap_mlp_gradients": (_i, [_vp, _vp, _vp, _i, _vp, ctypes.POINTER(ctypes.c_float)]),
    "sap_mlp_train": (_i, [_vp, _vp, _vp, _i, _i, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    "sap_mlp_last_error": (ctypes.c_char_p, []),
    "sap_solver_block_layout": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sap_options_default": (_i, [ctypes.POINTER(_COptions)]),
    "sap_banded_create": (_i, [_i, _i, _vp, _i, _pp]),
    "sap_banded_generate": (_i, [_i, _i, _d, _i, ctypes.c_uint64, _pp]),
    "sap_generate_band_host": (_i, [_i, _i, _d, _i, ctypes.c_uint64, _vp]),
    "sap_banded_copy_out": (_i, [_vp, _vp, _i]),
    "sap_banded_info": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sap_banded_destroy": (_i, [_vp]),
    "sap_csr_create": (_i, [_i, _i, _vp, _vp, _vp, _i, _pp]),
    "sap_csr_info": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sap_csr_destroy": (_i, [_vp]),
    "sap_spmv_banded_create": (_i, [_vp, _pp]),
    "sap_spmv_csr_create": (_i, [_vp, _pp]),
    "sap_spmv_callback_create": (_i, [_i, _vp, _vp, _pp]),
    "sap_spmv_apply": (_i, [_vp, _vp, _vp]),
    "sap_spmv_destroy": (_i, [_vp]),
    "sap_solver_create": (_i, [_i, ctypes.POINTER(_COptions), _i, _pp]),
    "sap_solver_destroy": (_i, [_vp]),
    "sap_solver_setup_banded": (_i, [_vp, _vp]),
    "sap_solver_setup_csr": (_i, [_vp, _vp]),
    "sap_solver_update": (_i, [_vp, _vp, ctypes.c_int64, _i, ctypes.POINTER(_i)]),
    "sap_solver_solve": (_i, [_vp, _vp, _vp, _vp, _i, ctypes.POINTER(_i)]),
    "sap_precond_apply": (_i, [_vp, _vp, _vp]),
    "sap_solver_get_stats": (_i, [_vp, ctypes.POINTER(_CStats)]),
    "sap_solver_get_monitor": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_char_p)]),
    "sap_solver_info": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "sap_solver_stream": (_vp, [_vp]),
    "sap_solver_get_reorder": (_i, [_vp, _i, _vp, ctypes.POINTER(ctypes.c_int64)]),
    "sap_reorder_host": (_i, [_i, _i, _vp, _vp, _vp, _i, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sap_reorder_host_stages": (_i, [_i, _vp, _vp, ctypes.POINTER(_i)]),
    "sap_blas_dots": (_i, [_i, _i, _pp, _pp, _vp, _vp]),
    "sap_blas_dots_noalloc": (_i, [_i, _i, _pp, _pp, _vp, _vp]),
    "sap_tc_gemm_batched": (_i, [_i, _i, _i, ctypes.c_float, _vp, _i, ctypes.c_longlong, _vp, _i, ctypes.c_longlong,
                                 ctypes.c_float, _vp, _i, ctypes.c_longlong, _i, _vp]),
    "sap_profile_select": (_i, [ctypes.c_char_p]),
    "sap_profile_read": (_i, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]),
}
for _name, (_res, _args) in _sig.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED_SYMBOLS = tuple(_sig)


def _check(code: int) -> None:
    if code == 0:
        return
    msg = (_lib.sap_last_error() or b"").decode()
    if -5 <= code <= -1:
        raise SystemError(code, msg)
    raise LibraryError(code, msg)


def _ptr(a):
    """(pointer, memspace) of a numpy array or a torch CUDA tensor (float64/int32)."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return ctypes.c_void_p(a.ctypes.data), HOST
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr()), DEVICE
    raise TypeError("expected a numpy array or a CUDA tensor")


def kernel_launch_count() -> int:
    """Number of kernels this library has enqueued since it was loaded."""
    return int(_lib.sap_kernel_launch_count())


def read_matrix_market(path: str):
    """CSR arrays (row_offsets int32, column_indices int32, values float64) and
    the shape of a Matrix Market coordinate matrix (the reference drivers'
    cusp::io::read_matrix_market_file); duplicates summed, rows and columns
    sorted.  Host-side only: pass the arrays to CsrMatrix for the device."""
    m, n, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    bp = path.encode()
    code = _lib.sap_mm_read_csr(bp, ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz), None, None, None)
    if code:
        raise LibraryError(code, (_lib.sap_mm_last_error() or b"").decode())
    rp = np.empty(m.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value, np.float64)
    code = _lib.sap_mm_read_csr(bp, ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz), rp.ctypes.data,
                                ci.ctypes.data, v.ctypes.data)
    if code:
        raise LibraryError(code, (_lib.sap_mm_last_error() or b"").decode())
    return rp, ci, v, (m.value, n.value)


def read_matrix_market_vector(path: str) -> np.ndarray:
    """A Matrix Market vector (array or one-column coordinate) as float64."""
    n = ctypes.c_int64()
    bp = path.encode()
    code = _lib.sap_mm_read_vector(bp, ctypes.byref(n), None)
    if code:
        raise LibraryError(code, (_lib.sap_mm_last_error() or b"").decode())
    out = np.empty(n.value, np.float64)
    code = _lib.sap_mm_read_vector(bp, ctypes.byref(n), out.ctypes.data)
    if code:
        raise LibraryError(code, (_lib.sap_mm_last_error() or b"").decode())
    return out


class _BatchResult(ctypes.Structure):
    _fields_ = [("rel_residual", ctypes.c_double), ("iterations", ctypes.c_float), ("converged", ctypes.c_int)]


def solve_batch(bands, ks, bs, num_partitions: int, opts: "Options", prec: str = "float"):
    """Solve independent banded systems (row-major bands as numpy arrays,
    half-bandwidths ks, right-hand sides bs) in one batched call; systems of
    equal half-bandwidth are solved together as one block-diagonal system to
    ||b_i - A_i x_i|| <= opts.relTol ||b_i|| each.  Returns (xs, results,
    seconds) with results[i] = (relative residual, iterations, converged)."""
    m = len(bands)
    ns = [len(b) for b in bs]
    bands = [np.ascontiguousarray(a, np.float64) for a in bands]
    bs = [np.ascontiguousarray(b, np.float64) for b in bs]
    xs = [np.zeros(n) for n in ns]
    n_arr = np.asarray(ns, np.int32)
    k_arr = np.asarray(ks, np.int32)
    pa = (ctypes.c_void_p * m)(*[a.ctypes.data for a in bands])
    pb = (ctypes.c_void_p * m)(*[b.ctypes.data for b in bs])
    px = (ctypes.c_void_p * m)(*[x.ctypes.data for x in xs])
    res = (_BatchResult * m)()
    sec = ctypes.c_double()
    copts = opts._c()
    _check(_lib.sap_batch_banded_solve(m, n_arr.ctypes.data, k_arr.ctypes.data, ctypes.cast(pa, ctypes.c_void_p),
                                       ctypes.cast(pb, ctypes.c_void_p), ctypes.cast(px, ctypes.c_void_p),
                                       int(num_partitions), ctypes.cast(ctypes.pointer(copts), ctypes.c_void_p),
                                       _PREC[prec], ctypes.cast(res, ctypes.c_void_p), ctypes.byref(sec)))
    return xs, [(r.rel_residual, r.iterations, bool(r.converged)) for r in res], sec.value


class _ReorderInfo(ctypes.Structure):
    _fields_ = [("K", ctypes.c_int), ("P", ctypes.c_int), ("k_db", ctypes.c_int), ("k_reorder", ctypes.c_int),
                ("var_band", ctypes.c_int), ("drop_actual", ctypes.c_double)]


def reorder_host(row_offsets, column_indices, values, num_partitions: int, opts: "Options" = None,
                 prec: str = "float", threads: int = 0) -> dict:
    """The host reordering of a CSR setup on its own, without a device
    (`sap_reorder_host`): DB, RCM, drop-off, second level and the composed
    permutations.  Returns K, P, k_db, k_reorder, var_band, drop_actual,
    the arrays dbRowPerm, finalPerm, finalReordering, first_rows, ks (the
    names of Solver.getReorder) and stage_ms (wall time of each stage,
    `sap_reorder_host_stages`)."""
    rp = np.ascontiguousarray(row_offsets, np.int32)
    ci = np.ascontiguousarray(column_indices, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    n, nnz, P = rp.size - 1, ci.size, int(num_partitions)
    if prec not in ("float", "double"):
        raise ValueError("prec must be 'float' or 'double'")
    copts = (opts or Options())._c()
    info = _ReorderInfo()
    out = {k: np.empty(m, np.int32) for k, m in (("dbRowPerm", n), ("finalPerm", n), ("finalReordering", n),
                                                  ("first_rows", max(P - 1, 0)), ("ks", P))}
    _check(_lib.sap_reorder_host(n, nnz, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, P,
                                 ctypes.cast(ctypes.pointer(copts), ctypes.c_void_p), _PREC[prec], int(threads),
                                 ctypes.cast(ctypes.pointer(info), ctypes.c_void_p),
                                 *[out[k].ctypes.data for k in ("dbRowPerm", "finalPerm", "finalReordering",
                                                                "first_rows", "ks")]))
    res = {f: getattr(info, f) for f, _ in _ReorderInfo._fields_}
    res["first_rows"] = out["first_rows"][:max(info.P - 1, 0)] if info.var_band else np.empty(0, np.int32)
    res["ks"] = out["ks"][:info.P]
    for k in ("dbRowPerm", "finalPerm", "finalReordering"):
        res[k] = out[k]
    cnt = _i(0)
    names, ms = (ctypes.c_char_p * 16)(), (ctypes.c_double * 16)()
    _check(_lib.sap_reorder_host_stages(16, ctypes.cast(names, ctypes.c_void_p), ctypes.cast(ms, ctypes.c_void_p),
                                        ctypes.byref(cnt)))
    res["stage_ms"] = {names[i].decode(): ms[i] for i in range(min(cnt.value, 16))}
    return res


def library_call_count() -> int:
    """Number of cuBLAS calls (wide-band batched GEMMs) since the library was loaded."""
    return int(_lib.sap_library_call_count())


def profile_select(kernel_name: str | None) -> None:
    """Bracket every launch of `kernel_name` with CUDA events on its stream."""
    _check(_lib.sap_profile_select((kernel_name or "").encode()))


def profile_read() -> tuple[float, int]:
    """(total milliseconds, launches) of the selected kernel since selection."""
    ms, cnt = ctypes.c_double(), ctypes.c_int64()
    _check(_lib.sap_profile_read(ctypes.byref(ms), ctypes.byref(cnt)))
    return ms.value, cnt.value


def blas_dots(xs, ys, out, stream: int = 0) -> None:
    """Fused FP64 dot products out[q] = xs[q] . ys[q] (q < 4) of CUDA tensors,
    through sap_blas_dots; `out` is a CUDA float64 tensor of len(xs)."""
    nq = len(xs)
    n = xs[0].numel()
    xa = (ctypes.c_void_p * nq)(*[t.data_ptr() for t in xs])
    ya = (ctypes.c_void_p * nq)(*[t.data_ptr() for t in ys])
    _check(_lib.sap_blas_dots(n, nq, xa, ya, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)))


def tc_gemm_batched(m: int, n: int, k: int, alpha: float, A, lda: int, sA: int, B, ldb: int, sB: int, beta: float,
                    C, ldc: int, sC: int, batch: int, stream: int = 0) -> None:
    """C_b = alpha A_b B_b + beta C_b on the tensor cores (TF32 inputs, FP32
    accumulation): the library's batched product of the wide-band
    factorization (sap_tc_gemm_batched).  A, B, C are CUDA float32 tensors or
    device addresses; the views are column-major with the given leading
    dimensions and batch strides (elements).  Waits for the stream."""
    def addr(t):
        return t if isinstance(t, int) else t.data_ptr()
    _check(_lib.sap_tc_gemm_batched(m, n, k, alpha, addr(A), lda, sA, addr(B), ldb, sB, beta, addr(C), ldc, sC,
                                    batch, stream or None))


def generate_band_host(n: int, k: int, d: float, dist: int = 1, seed: int = 0) -> np.ndarray:
    """Row-major band of BandedMatrix(n, k, d) generated on the host (no GPU)."""
    out = np.zeros(n * (2 * k + 1), dtype=np.float64)
    _check(_lib.sap_generate_band_host(n, k, float(d), dist, seed, ctypes.c_void_p(out.ctypes.data)))
    return out


# ---- Options / Stats ------------------------------------------------------------
_PREC = {"float": 0, "double": 1, "tf32": 2, "tf32_f16": 3}


@dataclass
class Options:
    """sap::Options (sap/solver.h:52-81), defaults of sap/solver.h:233-256."""
    solverType: int = BiCGStab2
    maxNumIterations: int = 100
    relTol: float = 1e-6
    absTol: float = 0.0
    testDB: bool = False
    isSPD: bool = False
    saveMem: bool = False
    performReorder: bool = True
    performDB: bool = True
    dbFirstStageOnly: bool = False
    applyScaling: bool = True
    maxBandwidth: int = 2**31 - 1
    gpuCount: int = 1
    dropOffFraction: float = 0.0
    factMethod: int = LU_only
    precondType: int = Spike
    safeFactorization: bool = False
    variableBandwidth: bool = True
    trackReordering: bool = False
    useBCR: bool = False
    ilu_level: int = -1
    # extension: FP64 refinement sweeps around BiCGStab(L) (0: the reference's solve)
    refinementSweeps: int = 0

    def _c(self) -> _COptions:
        c = _COptions()
        for f in fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, float(v) if isinstance(v, float) else int(v))
        return c


class Stats:
    """sap::Stats (sap/solver.h:89-140); times in milliseconds."""

    def __init__(self, c: _CStats):
        for name, _ in _CStats._fields_:
            setattr(self, name, getattr(c, name))

    def __repr__(self):
        keys = ("timeSetup", "timeSolve", "numIterations", "relResidualNorm", "bandwidth", "numPartitions")
        return "Stats(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in keys) + ")"


# ---- matrices -------------------------------------------------------------------
class BandedMatrix:
    """sap::BandedMatrix (sap/banded_matrix.h:25-95): a device-resident
    row-major FP64 band.  `BandedMatrix(n, k, d)` generates it like the
    reference (dist 0: rand() in [-10,10]); `BandedMatrix.from_array`
    wraps caller data."""

    def __init__(self, n: int, k: int, d: float, dist: int = 0, seed: int = 1, _handle=None):
        self.m_n = self.num_rows = self.num_cols = int(n)
        self.m_k = int(k)
        self.m_d = float(d)
        if _handle is None:
            h = ctypes.c_void_p()
            _check(_lib.sap_banded_generate(n, k, float(d), dist, seed, ctypes.byref(h)))
            _handle = h
        self._h = _handle
        self.num_entries = n * (2 * k + 1) - k * (k + 1)

    @classmethod
    def from_array(cls, band, n: int, k: int) -> "BandedMatrix":
        p, ms = _ptr(band)
        h = ctypes.c_void_p()
        _check(_lib.sap_banded_create(n, k, p, ms, ctypes.byref(h)))
        return cls(n, k, 0.0, _handle=h)

    def getBandedMatrix(self) -> np.ndarray:
        out = np.empty(self.m_n * (2 * self.m_k + 1), dtype=np.float64)
        _check(_lib.sap_banded_copy_out(self._h, ctypes.c_void_p(out.ctypes.data), HOST))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.sap_banded_destroy(h)
            self._h = None


class CsrMatrix:
    """Device CSR matrix, int32 indices and FP64 values (the reference's
    cusp::csr_matrix<int, double, device_memory>)."""

    def __init__(self, row_offsets, column_indices, values):
        rp = np.ascontiguousarray(row_offsets, dtype=np.int32)
        ci = np.ascontiguousarray(column_indices, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.num_rows = self.num_cols = rp.size - 1
        self.num_entries = ci.size
        h = ctypes.c_void_p()
        _check(_lib.sap_csr_create(self.num_rows, self.num_entries, ctypes.c_void_p(rp.ctypes.data),
                                   ctypes.c_void_p(ci.ctypes.data), ctypes.c_void_p(v.ctypes.data), HOST,
                                   ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.sap_csr_destroy(h)
            self._h = None


# ---- SpMV functors (sap/spmv.h) ---------------------------------------------------
class _Spmv:
    def __call__(self, v, Av):
        pv, msv = _ptr(v)
        pa, msa = _ptr(Av)
        if msv != DEVICE or msa != DEVICE:
            raise TypeError("SpMV operands must be CUDA tensors")
        _check(_lib.sap_spmv_apply(self._h, pv, pa))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.sap_spmv_destroy(h)
            self._h = None


class MVBanded(_Spmv):
    """MVBanded<Matrix> (sap/spmv.h:27-74)."""

    def __init__(self, A: BandedMatrix):
        self._A = A
        h = ctypes.c_void_p()
        _check(_lib.sap_spmv_banded_create(A._h, ctypes.byref(h)))
        self._h = h


class SpmvCusp(_Spmv):
    """SpmvCusp<Matrix> (sap/spmv.h:83-129): FP64 CSR product."""

    def __init__(self, A: CsrMatrix):
        self._A = A
        h = ctypes.c_void_p()
        _check(_lib.sap_spmv_csr_create(A._h, ctypes.byref(h)))
        self._h = h

    def getTime(self) -> float:
        return 0.0

    def getCount(self) -> float:
        return 0.0

    def getGFlops(self) -> float:
        return 0.0


# ---- Solver ------------------------------------------------------------------------
class Solver:
    """sap::Solver<Array, PrecValueType> (sap/solver.h:153-225).

    prec: the preconditioner's value type, "float" or "double" as the
    reference's PrecValueType, or the extensions "tf32" (FP32 storage, wide
    bands factored with TF32 tensor-core products) and "tf32_f16" (as "tf32",
    with FP16 block-scaled copies of the factor blocks for the sweeps)."""

    def __init__(self, numPartitions: int, opts: Options, prec: str = "float"):
        self._opts = opts
        h = ctypes.c_void_p()
        copts = opts._c()
        if prec not in _PREC:
            raise ValueError(f"prec must be one of {sorted(_PREC)}")
        _check(_lib.sap_solver_create(int(numPartitions), ctypes.byref(copts), _PREC[prec], ctypes.byref(h)))
        self._h = h

    def setup(self, A) -> bool:
        """Solver::setup(A) (sap/solver.h:339-404)."""
        self._A = A
        if isinstance(A, BandedMatrix):
            _check(_lib.sap_solver_setup_banded(self._h, A._h))
        elif isinstance(A, CsrMatrix):
            _check(_lib.sap_solver_setup_csr(self._h, A._h))
        else:
            raise TypeError("setup expects a BandedMatrix or a CsrMatrix")
        return True

    def update(self, entries) -> bool:
        """Solver::update(entries) (sap/solver.h:421-462)."""
        p, ms = _ptr(entries)
        acc = ctypes.c_int(1)
        n = entries.size if isinstance(entries, np.ndarray) else entries.numel()
        _check(_lib.sap_solver_update(self._h, p, n, ms, ctypes.byref(acc)))
        return bool(acc.value)

    def solve(self, spmv: _Spmv, b, x) -> bool:
        """Solver::solve(spmv, b, x) (sap/solver.h:477-562); x is the initial
        guess on entry and the solution on exit (numpy or CUDA tensor)."""
        pb, msb = _ptr(b)
        px, msx = _ptr(x)
        if msb != msx:
            raise TypeError("b and x must live in the same memory space")
        conv = ctypes.c_int(0)
        _check(_lib.sap_solver_solve(self._h, spmv._h, pb, px, msb, ctypes.byref(conv)))
        return bool(conv.value)

    def precond(self, v, z) -> None:
        """Precond::operator()(v, z) (sap/precond.h:1370-1386), CUDA tensors."""
        pv, _ = _ptr(v)
        pz, _ = _ptr(z)
        _check(_lib.sap_precond_apply(self._h, pv, pz))

    def getStats(self) -> Stats:
        c = _CStats()
        _check(_lib.sap_solver_get_stats(self._h, ctypes.byref(c)))
        return Stats(c)

    def getMonitorCode(self) -> int:
        code = ctypes.c_int()
        _check(_lib.sap_solver_get_monitor(self._h, ctypes.byref(code), None))
        return code.value

    def getMonitorMessage(self) -> str:
        msg = ctypes.c_char_p()
        _check(_lib.sap_solver_get_monitor(self._h, None, ctypes.byref(msg)))
        return (msg.value or b"").decode()

    def info(self):
        n, k, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.sap_solver_info(self._h, ctypes.byref(n), ctypes.byref(k), ctypes.byref(p)))
        return n.value, k.value, p.value

    def blockLayout(self):
        """(block size, blocks per partition, bytes per factor value read by the
        sweeps) of the wide-band block path; (0, 0, bytes) for the narrow band
        kernels."""
        bs, nb, vb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.sap_solver_block_layout(self._h, ctypes.byref(bs), ctypes.byref(nb), ctypes.byref(vb)))
        return bs.value, nb.value, vb.value

    REORDER_ARRAYS = ("dbRowPerm", "finalPerm", "finalReordering", "first_rows", "ks")

    def getReorder(self, name: str) -> np.ndarray:
        """Reordering results of a CSR setup (see sap_solver_get_reorder)."""
        w = self.REORDER_ARRAYS.index(name)
        cnt = ctypes.c_int64()
        _check(_lib.sap_solver_get_reorder(self._h, w, None, ctypes.byref(cnt)))
        out = np.empty(cnt.value, np.int32)
        if cnt.value:
            _check(_lib.sap_solver_get_reorder(self._h, w, ctypes.c_void_p(out.ctypes.data), ctypes.byref(cnt)))
        return out

    def stream(self) -> int:
        return _lib.sap_solver_stream(self._h) or 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.sap_solver_destroy(h)
            self._h = None


__all__ = ["Options", "Stats", "Solver", "BandedMatrix", "CsrMatrix", "MVBanded", "SpmvCusp", "SystemError",
           "LibraryError", "generate_band_host", "kernel_launch_count", "BiCGStab1", "BiCGStab2", "FGMRES", "LU_UL",
           "LU_only", "Spike", "Block", "NoPrecond", "EXPORTED_SYMBOLS"]
