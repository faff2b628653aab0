"""HBM throughput of the library's FP64 CSR SpMV (SpmvCusp,
k_spmv_csr_blocks) on the 1M-row reordered convection-diffusion matrix of
the benchmark workload.

    python -m saplibrary_b200.spmv_bench [--m 1000] [--reps 20]

Prints one JSON line: the best and median device time of y = A x over
`reps` launches (the library's CUDA events around the kernel on its
launching stream; before every launch the L2 is flushed by writing a 256 MB
buffer and then reading another, which leaves no dirty lines behind), the
algorithmic bytes of one
product, 12 nnz + 4 (n + 1) + 8 n (x) + 8 n (y): values and column indices,
row offsets, the source and the result vector, and the achieved GB/s
against the measured HBM copy bandwidth recorded in MEASURED_PEAKS.json
beside the repository; and the result's largest deviation from a numpy
product.
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
    ap.add_argument("--m", type=int, default=1000, help="grid side (n = m * m rows)")
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    import numpy as np
    import torch
    from . import CsrMatrix, SpmvCusp
    from .problems import convection_diffusion_csr, csr_matvec
    rp, ci, v, _ = convection_diffusion_csr(m=a.m, fill_reach=5 * a.m, seed=1)
    n, nnz = rp.size - 1, int(rp[-1])
    A = CsrMatrix(rp, ci, v)
    spmv = SpmvCusp(A)
    xh = np.random.default_rng(2).standard_normal(n)
    x = torch.tensor(xh, device="cuda")
    y = torch.empty_like(x)
    from . import profile_read, profile_select
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    clean = torch.ones(64 << 20, dtype=torch.float32, device="cuda")
    spmv(x, y)  # warm-up
    torch.cuda.synchronize()
    times = []
    for _ in range(a.reps):
        flush.fill_(1.0)
        clean.sum()
        torch.cuda.synchronize()
        profile_select("spmv_csr")
        spmv(x, y)
        ms, cnt = profile_read()
        profile_select(None)
        times.append(ms / max(cnt, 1))
    ref = csr_matvec(rp, ci, v, xh)
    err = float(np.abs(y.cpu().numpy() - ref).max() / np.abs(ref).max())
    bytes_ = 12 * nnz + 4 * (n + 1) + 16 * n
    peak, kind = _hbm_peak()
    best, med = min(times), sorted(times)[len(times) // 2]
    print(json.dumps({"kernel": "k_spmv_csr_blocks", "n": n, "nnz": nnz, "bytes": bytes_, "best_ms": best,
                      "median_ms": med, "gbs": bytes_ / best / 1e6, "frac_of_hbm": bytes_ / best / 1e6 / peak,
                      "peak_gbs": peak, "peak_source": kind, "max_rel_err_vs_numpy": err}), flush=True)


if __name__ == "__main__":
    main()
