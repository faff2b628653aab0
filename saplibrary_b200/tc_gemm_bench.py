"""Throughput of the library's tensor-core batched GEMM (sap_tc_gemm_batched)
on the product shapes of the wide-band block factorization.

    python -m saplibrary_b200.tc_gemm_bench [--shape M,N,K,BATCH ...] [--reps R] [--torch]

For each shape (column-major FP32 operands, TF32 products, FP32
accumulation) it prints one JSON line: the best device time over `reps`
calls (CUDA events on the calling stream; each call waits for its stream,
so the time is the kernel plus a small fixed host round trip), TFLOP/s
(2 M N K BATCH flops), the fraction of the measured dense bf16 tensor peak
recorded in MEASURED_PEAKS.json beside the repository (TF32 runs at half the
bf16 rate, so 0.5 of it is the TF32 ceiling), and with --torch the same
product through torch.bmm in TF32 mode (cuBLAS) for comparison.  Default
shapes: the 3168-row diagonal blocks of the 1M-row workload (16
partitions), their halves, and a 224-row block of the 2M-row K=200
workload (32 partitions).
"""
from __future__ import annotations

import argparse
import json
import os

DEFAULT_SHAPES = [(3168, 3168, 3168, 16), (1600, 1568, 1600, 16), (800, 800, 800, 16), (224, 224, 224, 32)]


def _peaks():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f).get("bf16_tflops"), "measured"
    except Exception:
        return 1590.0, "fallback"


def run(shape, reps: int, with_torch: bool) -> dict:
    import torch
    from . import _lib, tc_gemm_batched
    m, n, k, b = shape
    A = torch.randn(b, k, m, device="cuda")  # per batch element: m x k column-major
    B = torch.randn(b, n, k, device="cuda")  # k x n column-major
    C = torch.zeros(b, n, m, device="cuda")  # m x n column-major
    stream = torch.cuda.current_stream().cuda_stream
    tc_gemm_batched(m, n, k, 1.0, A, m, m * k, B, k, k * n, 0.0, C, m, m * n, b, stream)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        rc = _lib.sap_tc_gemm_batched(m, n, k, 1.0, A.data_ptr(), m, m * k, B.data_ptr(), k, k * n, 0.0,
                                      C.data_ptr(), m, m * n, b, stream)
        e1.record()
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError(f"sap_tc_gemm_batched returned {rc}")
        best = min(best, e0.elapsed_time(e1))
    flops = 2.0 * m * n * k * b
    peak, kind = _peaks()
    out = {"shape": [m, n, k, b], "ms": best, "tflops": flops / best / 1e9,
           "frac_of_bf16_peak": flops / best / 1e9 / peak, "peak_bf16_tflops": peak, "peak_source": kind}
    if with_torch:
        torch.backends.cuda.matmul.allow_tf32 = True
        At, Bt = A.transpose(1, 2), B.transpose(1, 2)
        R = torch.bmm(At, Bt)
        tb = float("inf")
        for _ in range(reps):
            e0.record()
            R = torch.bmm(At, Bt)
            e1.record()
            torch.cuda.synchronize()
            tb = min(tb, e0.elapsed_time(e1))
        out["torch_tf32_ms"] = tb
        out["torch_tf32_tflops"] = flops / tb / 1e9
        out["max_abs_diff_vs_torch"] = float((C.transpose(1, 2) - R).abs().max())
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--shape", action="append", default=None, help="M,N,K,BATCH (repeatable)")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--torch", action="store_true", help="also time torch.bmm in TF32 mode")
    a = ap.parse_args()
    shapes = [tuple(int(v) for v in s.split(",")) for s in a.shape] if a.shape else DEFAULT_SHAPES
    for shp in shapes:
        print(json.dumps(run(shp, a.reps, a.torch)), flush=True)


if __name__ == "__main__":
    main()
