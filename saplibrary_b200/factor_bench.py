"""Device time of the narrow-band partition factorisation (the LU and, for
LU_UL, the mirrored UL of every partition in one launch) on a generated
banded matrix, for the panel-blocked kernel (k_factor_panel, the default for
half-bandwidths up to 120) and the one-pivot-at-a-time ring kernel it
replaced (k_factor_smem, SAPB_FACTOR_KERNEL=ring).

    python -m saplibrary_b200.factor_bench [--n 200000] [--k 50] [--p 10]
        [--prec double] [--reps 5] [--kernels panel,ring]

Prints one JSON line per kernel: the best device time of the factor launch
over `reps` setups (the library's CUDA events around the kernel on its
launching stream), the time per pivot of one partition, and the
factorisation's algorithmic HBM traffic (each band column read and written
once: 2 (2K + 1) n elements, LU and UL counted separately) against the
measured HBM copy bandwidth recorded in MEASURED_PEAKS.json beside the
repository.  The factor is a serial chain of n / P pivots per partition, so
it is bound by that chain's latency, not by HBM; the fraction shows how far.
"""
from __future__ import annotations

import argparse
import json
import os


def _hbm_peak():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=200000)
    ap.add_argument("--k", type=int, default=50)
    ap.add_argument("--p", type=int, default=10)
    ap.add_argument("--prec", default="double", choices=["double", "float"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--kernels", default="panel,ring")
    a = ap.parse_args()
    from . import LU_UL, BandedMatrix, Options, Solver, profile_read, profile_select
    A = BandedMatrix(a.n, a.k, 1.0, dist=1, seed=1)
    peak, kind = _hbm_peak()
    esize = 8 if a.prec == "double" else 4
    jobs = 2 * a.p - 2  # LU_UL: the LU of partitions 0..P-2 and the UL of partitions 1..P-1
    for kern in a.kernels.split(","):
        if kern == "ring":
            os.environ["SAPB_FACTOR_KERNEL"] = "ring"
        else:
            os.environ.pop("SAPB_FACTOR_KERNEL", None)
        s = Solver(a.p, Options(performReorder=False, variableBandwidth=False, applyScaling=False,
                                factMethod=LU_UL), prec=a.prec)
        s.setup(A)
        best = float("inf")
        for _ in range(a.reps):
            profile_select("factor")
            s.setup(A)
            ms, cnt = profile_read()
            profile_select(None)
            best = min(best, ms / max(cnt, 1))
        os.environ.pop("SAPB_FACTOR_KERNEL", None)
        rows = a.n // a.p
        traffic = 2 * (2 * a.k + 1) * rows * jobs * esize
        print(json.dumps({"kernel": "k_factor_panel" if kern == "panel" else "k_factor_smem", "n": a.n, "K": a.k,
                          "P": a.p, "prec": a.prec, "best_ms": best, "ns_per_pivot": best * 1e6 / rows,
                          "traffic_bytes": traffic, "gbs": traffic / best / 1e6,
                          "frac_of_hbm": traffic / best / 1e6 / peak, "peak_gbs": peak, "peak_source": kind}),
              flush=True)
        del s


if __name__ == "__main__":
    main()
