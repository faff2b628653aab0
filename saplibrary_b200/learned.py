"""Learned solver settings: small MLPs (16 features -> 64 -> 64 -> one logit
per setting) that pick the solver settings for a matrix, trained on the GPU by
this library's kernels (`sap_mlp_*`) from the outcomes the solver itself
produces when swept over those settings.  The setting used without the
network (the default heuristic) is each family's `default`, and the chooser
falls back to it where the network is unsure.  Two families:

* `BANDED`: banded matrices (no reordering).  Settings: partition count
  P in {1, 4, 16, 64}; coupled (SPIKE) with LU_UL or LU_only, or decoupled
  (block-Jacobi).  Features: `band_features` (size, bandwidth, diagonal
  dominance, decay of the off-diagonal magnitudes, sign mix).
* `SPARSE`: sparse matrices set up with the DB / RCM / drop-off reordering
  (the stencil + fill family of the 1M-row workload, at smaller sizes).
  Settings: P in {4, 16, 64}; coupled or decoupled; drop-off fraction in
  {0, 1e-4, 1e-2}.  Features: `csr_features` (size, nonzero profile,
  dominance of each row's largest entry, and the bandwidths after DB and
  after RCM from the host reordering, `reorder_host`).

    X, T = sweep(BANDED, count, seed)              # features, measured times
    net = SettingsNet(BANDED); net.train(X, labels_from_times(T))
    pick = net.choose(X)                           # index into BANDED.settings
    gain(BANDED, T, pick)                          # against the default

Labels are the settings with the lowest measured time-to-solution (setup +
flexible GMRES with an FP32 preconditioner to relres 1e-10, best of a few
repetitions); a setting that fails or does not converge costs infinity.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import (Block, BandedMatrix, CsrMatrix, FGMRES, LU_UL, LU_only, LibraryError, MVBanded, Options, Solver,
               Spike, SpmvCusp, _check, _lib, reorder_host)

NUM_FEATURES = 16
# below this largest class probability the chooser keeps the default setting
CONFIDENCE = 0.5


@dataclass(frozen=True)
class Family:
    """A matrix family: its settings (partitions, preconditioner type,
    factorisation method, drop-off fraction) and the default one."""
    name: str
    settings: tuple
    default: int


BANDED = Family("banded", (
    (1, Spike, LU_UL, 0.0), (4, Spike, LU_UL, 0.0), (16, Spike, LU_UL, 0.0), (64, Spike, LU_UL, 0.0),
    (4, Spike, LU_only, 0.0), (16, Spike, LU_only, 0.0), (64, Spike, LU_only, 0.0),
    (4, Block, LU_UL, 0.0), (16, Block, LU_UL, 0.0), (64, Block, LU_UL, 0.0)), default=2)
_SPARSE_SETTINGS = tuple((P, pt, LU_UL, dr) for P in (4, 16, 64) for pt in (Spike, Block) for dr in (0.0, 1e-4, 1e-2))
SPARSE = Family("sparse", _SPARSE_SETTINGS, default=_SPARSE_SETTINGS.index((16, Spike, LU_UL, 1e-4)))

# the banded family under its earlier names
SETTINGS = BANDED.settings
DEFAULT_SETTING = BANDED.default


def band_features(band: np.ndarray, n: int, K: int) -> np.ndarray:
    """16 features of a banded matrix given as its row-major band (n x
    (2K+1), element (i, j) at [i, K + j - i]): size and bandwidth, diagonal
    dominance statistics, decay of the off-diagonal magnitudes with the
    distance from the diagonal, sign mix."""
    B = np.asarray(band, dtype=np.float64).reshape(n, 2 * K + 1)
    diag = np.abs(B[:, K])
    off = np.abs(B).sum(axis=1) - diag
    dom = diag / np.maximum(off, 1e-300)
    mag = np.abs(B).mean(axis=0)  # mean magnitude per distance (-K..K)
    dmean = max(diag.mean(), 1e-300)

    def at(d):
        return 0.5 * (mag[K + d] + mag[K - d]) / dmean

    outer = np.abs(B[:, :K // 2 + 1]).sum() + np.abs(B[:, K + K // 2 + (K % 2):]).sum()
    offsum = max(off.sum(), 1e-300)
    f = [
        math.log10(n), math.log10(max(K, 1)), 1000.0 * K / n, float(dom.min()), float(dom.mean()),
        float(dom.std()), float(outer / offsum), at(1) if K >= 1 else 0.0, at(max(K // 4, 1)), at(max(K // 2, 1)),
        at(K), math.log10(n * (2 * K + 1)), float((np.sign(B[:, np.arange(2 * K + 1) != K]) < 0).mean()),
        float(diag.std() / dmean), math.log10(n / max(K, 1)), float((dom < 1.0).mean()),
    ]
    return np.asarray(f, dtype=np.float32)


def csr_features(rp: np.ndarray, ci: np.ndarray, v: np.ndarray) -> np.ndarray:
    """16 features of a sparse matrix (CSR): size, nonzero profile, how much
    each row's largest entry dominates it (rows may be permuted, so the
    diagonal is not known before the DB matching), value spread and signs,
    and the bandwidths after DB and after RCM of the host reordering."""
    n = rp.size - 1
    nnz = int(rp[-1])
    cnt = np.diff(rp).astype(np.float64)
    a = np.abs(np.asarray(v, np.float64))
    rows = np.repeat(np.arange(n), np.diff(rp))
    rmax = np.zeros(n)
    np.maximum.at(rmax, rows, a)
    rsum = np.bincount(rows, weights=a, minlength=n)
    dom = rmax / np.maximum(rsum - rmax, 1e-300)
    info = reorder_host(rp, ci, v, 16, Options(dropOffFraction=0.0))
    kdb, kre = max(int(info["k_db"]), 1), max(int(info["k_reorder"]), 1)
    med = float(np.median(a / np.maximum(rmax[rows], 1e-300)))
    f = [
        math.log10(n), nnz / n, float(cnt.max()), math.log10(kdb), math.log10(kre), 1000.0 * kre / n,
        float(dom.min()), float(dom.mean()), float(dom.std()), float((dom > 1.0).mean()), med,
        math.log10(max(nnz, 1)), kre / kdb, float((np.asarray(v) < 0).mean()), math.log10(n / kre),
        float(cnt.std()),
    ]
    return np.asarray(f, dtype=np.float32)


def _time_solves(make_solver, setup_arg, spmv, b, reps: int) -> float:
    import torch
    bd = torch.tensor(b, device="cuda")
    best = math.inf
    try:
        s = make_solver()
    except LibraryError:
        return best
    for _ in range(reps):
        x = torch.zeros_like(bd)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            s.setup(setup_arg)
            ok = s.solve(spmv, bd, x)
        except LibraryError:
            ok = False
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        if ok:
            best = min(best, t)
    return best


def measure(band: np.ndarray, n: int, K: int, setting: int, b: np.ndarray, reps: int = 3,
            rel_tol: float = 1e-10) -> float:
    """Time-to-solution (s) of setup + FGMRES solve of a banded matrix with
    an FP32 preconditioner under BANDED.settings[setting] (best of `reps`,
    so that a host stall in one repetition does not enter the label); inf
    when the solve fails or does not converge."""
    P, ptype, fact, _ = BANDED.settings[setting]
    opts = Options(solverType=FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                   factMethod=fact, precondType=ptype, relTol=rel_tol, maxNumIterations=300)
    A = BandedMatrix.from_array(band, n, K)
    return _time_solves(lambda: Solver(P, opts, prec="float"), A, MVBanded(A), b, reps)


def measure_sparse(A: CsrMatrix, setting: int, b: np.ndarray, reps: int = 2, rel_tol: float = 1e-10) -> float:
    """As `measure`, for a CSR matrix set up with the reordering under
    SPARSE.settings[setting]."""
    P, ptype, fact, drop = SPARSE.settings[setting]
    opts = Options(solverType=FGMRES, dropOffFraction=drop, factMethod=fact, precondType=ptype, relTol=rel_tol,
                   maxNumIterations=300)
    return _time_solves(lambda: Solver(P, opts, prec="float"), A, SpmvCusp(A), b, reps)


def random_band(rng: np.random.Generator, n_range=(20000, 200000), k_range=(10, 120), d_range=(0.5, 1.5)):
    """A banded test matrix of the configs' families: N log-uniform, K and
    the dominance d uniform, off-diagonals U[-1,1] or N(0,1)."""
    from . import generate_band_host
    n = int(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]))))
    K = int(rng.integers(k_range[0], k_range[1] + 1))
    d = float(rng.uniform(*d_range))
    dist = int(rng.choice([1, 2]))
    band = generate_band_host(n, K, d, dist, seed=int(rng.integers(1 << 31)))
    return band, n, K


def random_sparse(rng: np.random.Generator, m_range=(60, 160)):
    """A matrix of the stencil + fill family (convection-diffusion on an
    m x m grid, random fill, rows permuted): m uniform, convection, fill
    count, reach and magnitude drawn per matrix."""
    from .problems import convection_diffusion_csr
    m = int(rng.integers(m_range[0], m_range[1] + 1))
    rp, ci, v, _ = convection_diffusion_csr(m=m, conv=float(rng.uniform(0.1, 0.8)),
                                            fill_per_row=int(rng.integers(1, 4)),
                                            fill_reach=int(m * rng.uniform(1.0, 8.0)),
                                            fill_mag=float(rng.uniform(0.02, 0.3)), seed=int(rng.integers(1 << 31)))
    return rp, ci, v


def sweep(family, count: int | None = None, seed: int = 0, **kw) -> tuple[np.ndarray, np.ndarray]:
    """Features [count, 16] and measured time-to-solution [count, settings]
    of `count` seeded matrices of the family (BANDED or SPARSE; an integer
    first argument is read as the banded family's count, the earlier form)."""
    if not isinstance(family, Family):
        family, count = BANDED, family
    rng = np.random.default_rng(seed)
    X, T = [], []
    for _ in range(count):
        if family is BANDED:
            band, n, K = random_band(rng, **kw)
            b = np.random.default_rng(n + K).standard_normal(n)
            X.append(band_features(band, n, K))
            T.append([measure(band, n, K, s, b) for s in range(len(family.settings))])
        else:
            rp, ci, v = random_sparse(rng, **kw)
            n = rp.size - 1
            b = np.random.default_rng(n).standard_normal(n)
            X.append(csr_features(rp, ci, v))
            A = CsrMatrix(rp, ci, v)
            T.append([measure_sparse(A, s, b) for s in range(len(family.settings))])
    return np.asarray(X, np.float32), np.asarray(T, np.float64)


class SettingsNet:
    """The MLP on the GPU (sap_mlp_*), with feature standardisation."""

    def __init__(self, family: Family = BANDED, hidden=(64, 64), seed: int = 7):
        if not isinstance(family, Family):  # the earlier form SettingsNet(seed=...) passed by keyword only
            raise TypeError("family must be BANDED or SPARSE")
        self.family = family
        h = ctypes.c_void_p()
        _check(_lib.sap_mlp_create(NUM_FEATURES, hidden[0], hidden[1], len(family.settings), seed, ctypes.byref(h)))
        self._h = h
        self.mu = np.zeros(NUM_FEATURES, np.float32)
        self.sd = np.ones(NUM_FEATURES, np.float32)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.sap_mlp_destroy(h)
            self._h = None

    def _norm(self, X):
        return np.ascontiguousarray((np.asarray(X, np.float32) - self.mu) / self.sd, np.float32)

    def params(self) -> np.ndarray:
        out = np.empty(_lib.sap_mlp_num_params(self._h), np.float32)
        _check(_lib.sap_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check(_lib.sap_mlp_set_params(self._h, p.ctypes.data))

    def logits(self, X, normalise: bool = True) -> np.ndarray:
        Xn = self._norm(X) if normalise else np.ascontiguousarray(X, np.float32)
        out = np.empty((Xn.shape[0], len(self.family.settings)), np.float32)
        _check(_lib.sap_mlp_forward(self._h, Xn.ctypes.data, Xn.shape[0], out.ctypes.data))
        return out

    def gradients(self, X, labels, normalise: bool = False):
        Xn = self._norm(X) if normalise else np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        g = np.empty(_lib.sap_mlp_num_params(self._h), np.float32)
        loss = ctypes.c_float()
        _check(_lib.sap_mlp_gradients(self._h, Xn.ctypes.data, y.ctypes.data, Xn.shape[0], g.ctypes.data,
                                      ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, labels, epochs: int = 400, lr: float = 3e-3) -> float:
        X = np.asarray(X, np.float32)
        self.mu = X.mean(axis=0)
        self.sd = np.maximum(X.std(axis=0), 1e-6).astype(np.float32)
        Xn = self._norm(X)
        y = np.ascontiguousarray(labels, np.int32)
        loss = ctypes.c_float()
        _check(_lib.sap_mlp_train(self._h, Xn.ctypes.data, y.ctypes.data, Xn.shape[0], epochs, lr, ctypes.byref(loss)))
        return loss.value

    def probabilities(self, X) -> np.ndarray:
        z = self.logits(X).astype(np.float64)
        z -= z.max(axis=1, keepdims=True)
        e = np.exp(z)
        return e / e.sum(axis=1, keepdims=True)

    def choose(self, X, min_confidence: float = CONFIDENCE) -> np.ndarray:
        """The setting of the largest logit per matrix; the default heuristic
        where the network is unsure (largest probability below
        `min_confidence`), so that a matrix unlike the training set falls
        back to the method without the network."""
        p = self.probabilities(X)
        picks = p.argmax(axis=1)
        picks[p.max(axis=1) < min_confidence] = self.family.default
        return picks


def labels_from_times(T: np.ndarray) -> np.ndarray:
    """The fastest setting per matrix."""
    return np.argmin(T, axis=1).astype(np.int32)


def gain(*args) -> dict:
    """gain(family, T, picks) (or gain(T, picks) for the banded family):
    total time-to-solution of the picked settings against the family's
    default setting and the per-matrix best, over the matrices of T."""
    family, T, picks = (args if len(args) == 3 else (BANDED,) + args)
    rows = np.arange(T.shape[0])
    chosen = T[rows, picks]
    default = T[:, family.default]
    best = T.min(axis=1)
    finite = np.isfinite(chosen) & np.isfinite(default)
    return {"total_chosen_s": float(chosen[finite].sum()), "total_default_s": float(default[finite].sum()),
            "total_best_s": float(best[finite].sum()), "failed_chosen": int((~np.isfinite(chosen)).sum()),
            "failed_default": int((~np.isfinite(default)).sum()),
            "speedup_vs_default": float(default[finite].sum() / max(chosen[finite].sum(), 1e-30)),
            "picked_best": float((picks == np.argmin(T, axis=1)).mean())}


def evaluate(family: Family, train: int, held: int, seed: int, **kw) -> dict:
    """Sweep train + held matrices of the family, train on the first
    `train`, report the held-out gain over the default setting."""
    X, T = sweep(family, train + held, seed, **kw)
    net = SettingsNet(family, seed=seed)
    loss = net.train(X[:train], labels_from_times(T[:train]), epochs=600)
    g = gain(family, T[train:], net.choose(X[train:]))
    g.update({"family": family.name, "train": train, "held_out": held, "final_train_loss": loss,
              "settings": len(family.settings), "default_setting": list(family.settings[family.default])})
    return g


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="measured settings sweep, training and held-out gain")
    ap.add_argument("--family", default="banded", choices=["banded", "sparse"])
    ap.add_argument("--train", type=int, default=160)
    ap.add_argument("--held", type=int, default=40)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args()
    if a.family == "banded":
        print(json.dumps(evaluate(BANDED, a.train, a.held, a.seed, n_range=(20000, 200000), k_range=(10, 150),
                                  d_range=(0.5, 1.5))))
    else:
        print(json.dumps(evaluate(SPARSE, a.train, a.held, a.seed, m_range=(60, 200))))
