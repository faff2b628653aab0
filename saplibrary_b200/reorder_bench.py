"""Host time of the sparse setup's reordering stages (DB, RCM, drop-off,
coupling split, second-level reordering, variable-band widths, composed
permutations) on the 1M-row convection-diffusion workload, through
`sap_reorder_host` (no device needed).

    python -m saplibrary_b200.reorder_bench [--m 1000] [--threads 0]
        [--reps 5] [--prec float]

The matrix is the bench's sparse workload: an m x m 5-point
convection-diffusion grid (convection 0.3) with 2 fill entries per row
within +-5,000 of the diagonal, rows permuted; 16 partitions, drop-off
1e-4.  Prints one JSON line: the best and median wall time of the whole
call over `reps` calls after one warm-up (the pipeline keeps no memory
between calls here, so every call also faults in its scratch) and the
median time of every stage as the pipeline reports it
(`sap_reorder_host_stages`).  The stages run the same code as a solver
setup; the call adds the conversion of the input and the DB weights
computed on the host (a setup computes them on the device).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import time


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=1000)
    ap.add_argument("--threads", type=int, default=0, help="host threads (0: the OpenMP default)")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--prec", default="float", choices=["float", "double"])
    a = ap.parse_args()

    import saplibrary_b200 as sap
    from saplibrary_b200.problems import convection_diffusion_csr

    rp, ci, v, _ = convection_diffusion_csr(m=a.m, conv=0.3, fill_per_row=2, fill_reach=5 * a.m, fill_mag=0.1, seed=0)
    opts = sap.Options(dropOffFraction=1e-4)
    sap.reorder_host(rp, ci, v, 16, opts, prec=a.prec, threads=a.threads)  # warm-up
    walls, stages, r = [], {}, None
    for _ in range(a.reps):
        t0 = time.perf_counter()
        r = sap.reorder_host(rp, ci, v, 16, opts, prec=a.prec, threads=a.threads)
        walls.append((time.perf_counter() - t0) * 1e3)
        for k, t in r["stage_ms"].items():
            stages.setdefault(k, []).append(t)
    print(json.dumps({
        "workload": f"cd2d_m{a.m}_conv0.3_fill2x{5 * a.m}_rowperm_p16_drop1e-4", "n": int(rp.size - 1),
        "nnz": int(ci.size), "prec": a.prec, "threads": a.threads or os.cpu_count(), "reps": a.reps,
        "call_ms_best": round(min(walls), 2), "call_ms_median": round(statistics.median(walls), 2),
        "stage_ms_median": {k: round(statistics.median(t), 2) for k, t in stages.items()},
        "K": r["K"], "P": r["P"], "k_db": r["k_db"], "k_reorder": r["k_reorder"],
    }))


if __name__ == "__main__":
    main()
