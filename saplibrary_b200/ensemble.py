"""Batched ensemble of independent banded systems: the batched solve
(`solve_batch`, one block-diagonal stack per half-bandwidth) against solving
the systems one by one with the same options.

Ensemble (seeded): `count` systems, N log-uniform in [n_min, n_max], K drawn
uniformly from `ks`, dominance d uniform in [0.8, 1.2], off-diagonals
U[-1,1] (diagonal d times the row sum of their magnitudes), b ~ N(0,1).

    python -m saplibrary_b200.ensemble --count 512
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import (BandedMatrix, FGMRES, LU_UL, MVBanded, Options, Solver, generate_band_host, solve_batch)


def make_ensemble(count: int, seed: int, n_min=2000, n_max=200000, ks=(8, 16, 32, 64, 128)):
    rng = np.random.default_rng(seed)
    bands, kk, bs = [], [], []
    for _ in range(count):
        n = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        K = int(rng.choice(ks))
        K = min(K, n // 4)
        d = float(rng.uniform(0.8, 1.2))
        bands.append(generate_band_host(n, K, d, 1, seed=int(rng.integers(1 << 31))))
        kk.append(K)
        bs.append(rng.standard_normal(n))
    return bands, kk, bs


def options(rel_tol=1e-10):
    return Options(solverType=FGMRES, performReorder=False, variableBandwidth=False, applyScaling=False,
                   factMethod=LU_UL, relTol=rel_tol, maxNumIterations=400)


def one_by_one(bands, ks, bs, P, prec="float"):
    """Per-system wall times (s) and relative residuals, each system solved
    on its own (host arrays in and out, as the batch)."""
    times, rels = [], []
    for band, K, b in zip(bands, ks, bs):
        n = len(b)
        t0 = time.perf_counter()
        A = BandedMatrix.from_array(band, n, K)
        s = Solver(P, options(), prec=prec)
        s.setup(A)
        x = np.zeros(n)
        s.solve(MVBanded(A), b, x)
        times.append(time.perf_counter() - t0)
        rels.append(s.getStats().relResidualNorm)
    return np.asarray(times), np.asarray(rels)


def run(count=512, seed=3, P=8, prec="float", reps=1, **kw) -> dict:
    """Both legs `reps` times: the batched time is the best batch, the one by
    one times the best of each system (host stalls on a shared machine hit
    single repetitions)."""
    bands, ks, bs = make_ensemble(count, seed, **kw)
    solve_batch(bands[:4], ks[:4], bs[:4], P, options(), prec)  # warm-up
    secs = []
    for _ in range(reps):
        xs, res, sec = solve_batch(bands, ks, bs, P, options(), prec)
        secs.append(sec)
    sec = min(secs)
    rel = np.asarray([r[0] for r in res])
    t1 = None
    for _ in range(reps):
        t, rel1 = one_by_one(bands, ks, bs, P, prec)
        t1 = t if t1 is None else np.minimum(t1, t)
    return {
        "systems": count, "rows": int(sum(len(b) for b in bs)), "reps": reps, "batched_s": sec,
        "batched_s_all": [round(v, 4) for v in secs],
        "batched_solves_per_s": count / sec, "batched_max_rel_residual": float(rel.max()),
        "batched_all_converged": bool(all(r[2] for r in res)),
        "one_by_one_s": float(t1.sum()), "one_by_one_solves_per_s": count / float(t1.sum()),
        "one_by_one_p50_s": float(np.percentile(t1, 50)), "one_by_one_p99_s": float(np.percentile(t1, 99)),
        "one_by_one_max_rel_residual": float(rel1.max()),
        "speedup": float(t1.sum()) / sec,
        "note": "batched: every system completes with its stack, per-system time = batch time",
    }


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--parts", type=int, default=8)
    ap.add_argument("--prec", default="float")
    a = ap.parse_args()
    print(json.dumps(run(a.count, a.seed, a.parts, a.prec)))
