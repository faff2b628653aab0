"""Learned solver settings: a small MLP (16 features -> 64 -> 64 -> one logit
per setting) that picks the partition count and the coupled (SPIKE) or
decoupled (block-Jacobi) preconditioner for a banded matrix, trained on the
GPU by this library's kernels (`sap_mlp_*`) from the outcomes the solver
itself produces when swept over those settings.  The default heuristic (the
setting used without the network) is `DEFAULT_SETTING`.

    feats = band_features(band, n, K)           # host, numpy
    table = sweep(bands, ...)                   # measured time-to-solution per setting
    net = SettingsNet(); net.train(X, labels)   # GPU kernels
    pick = net.choose(X)                        # index into SETTINGS
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import (BandedMatrix, Block, FGMRES, LU_UL, LibraryError, MVBanded, Options, Solver, Spike, _check, _lib)

# settings the network chooses from: (partitions, preconditioner type)
SETTINGS = [(1, Spike), (4, Spike), (16, Spike), (64, Spike), (4, Block), (16, Block), (64, Block)]
DEFAULT_SETTING = 2  # 16 partitions, coupled SPIKE
NUM_FEATURES = 16
# below this largest class probability the chooser keeps the default setting
CONFIDENCE = 0.5


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


def measure(band: np.ndarray, n: int, K: int, setting: int, b: np.ndarray, reps: int = 3,
            rel_tol: float = 1e-10) -> float:
    """Time-to-solution (s) of setup + FGMRES solve with an FP32
    preconditioner under one setting (best of `reps`, so that a host stall
    in one repetition does not enter the label); inf when the solve does
    not converge."""
    import torch
    P, ptype = SETTINGS[setting]
    opts = Options(solverType=FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                   factMethod=LU_UL, precondType=ptype, relTol=rel_tol, maxNumIterations=300)
    A = BandedMatrix.from_array(band, n, K)
    spmv = MVBanded(A)
    bd = torch.tensor(b, device="cuda")
    best = math.inf
    s = Solver(P, opts, prec="float")
    for _ in range(reps):
        x = torch.zeros_like(bd)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            s.setup(A)
            ok = s.solve(spmv, bd, x)
        except LibraryError:
            ok = False
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        if ok:
            best = min(best, t)
    return best


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


def sweep(count: int, seed: int, **family) -> tuple[np.ndarray, np.ndarray]:
    """Features [count, 16] and measured time-to-solution [count, settings]."""
    from . import generate_band_host  # noqa: F401
    rng = np.random.default_rng(seed)
    X, T = [], []
    for _ in range(count):
        band, n, K = random_band(rng, **family)
        b = np.random.default_rng(n + K).standard_normal(n)
        X.append(band_features(band, n, K))
        T.append([measure(band, n, K, s, b) for s in range(len(SETTINGS))])
    return np.asarray(X, np.float32), np.asarray(T, np.float64)


class SettingsNet:
    """The MLP on the GPU (sap_mlp_*), with feature standardisation."""

    def __init__(self, hidden=(64, 64), seed: int = 7):
        h = ctypes.c_void_p()
        _check(_lib.sap_mlp_create(NUM_FEATURES, hidden[0], hidden[1], len(SETTINGS), seed, ctypes.byref(h)))
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
        out = np.empty((Xn.shape[0], len(SETTINGS)), np.float32)
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
        picks[p.max(axis=1) < min_confidence] = DEFAULT_SETTING
        return picks


def labels_from_times(T: np.ndarray) -> np.ndarray:
    """The fastest setting per matrix."""
    return np.argmin(T, axis=1).astype(np.int32)


def gain(T: np.ndarray, picks: np.ndarray) -> dict:
    """Total time-to-solution of the picked settings against the default
    setting and the per-matrix best, over the matrices of T."""
    rows = np.arange(T.shape[0])
    chosen = T[rows, picks]
    default = T[:, DEFAULT_SETTING]
    best = T.min(axis=1)
    finite = np.isfinite(chosen) & np.isfinite(default)
    return {"total_chosen_s": float(chosen[finite].sum()), "total_default_s": float(default[finite].sum()),
            "total_best_s": float(best[finite].sum()), "failed_chosen": int((~np.isfinite(chosen)).sum()),
            "failed_default": int((~np.isfinite(default)).sum()),
            "speedup_vs_default": float(default[finite].sum() / max(chosen[finite].sum(), 1e-30)),
            "picked_best": float((picks == np.argmin(T, axis=1)).mean())}


def evaluate(train: int, held: int, seed: int, **family) -> dict:
    """Sweep train + held matrices, train on the first `train`, report the
    held-out gain over the default setting."""
    X, T = sweep(train + held, seed, **family)
    net = SettingsNet(seed=seed)
    loss = net.train(X[:train], labels_from_times(T[:train]), epochs=600)
    g = gain(T[train:], net.choose(X[train:]))
    g.update({"train": train, "held_out": held, "final_train_loss": loss, "settings": len(SETTINGS),
              "default_setting": SETTINGS[DEFAULT_SETTING][0]})
    return g


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="measured settings sweep, training and held-out gain")
    ap.add_argument("--train", type=int, default=160)
    ap.add_argument("--held", type=int, default=40)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args()
    print(json.dumps(evaluate(a.train, a.held, a.seed, n_range=(20000, 200000), k_range=(10, 150),
                              d_range=(0.5, 1.5))))
