"""Benchmark of the SPIKE-preconditioned BiCGStab(2) solve on B200.

One step = one time-to-solution of the named workload: preconditioner
setup (band conversion, partitioned LU/UL factorisation, spike tips,
reduced system, sweep transfer matrices) plus the BiCGStab(2) solve to
FP64 relative residual 1e-10, as Solver::setup + Solver::solve of the
reference (sap/solver.h:339-562).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  With N > 1 (torchrun) every rank solves its
own independent system (replicas; the solve does not shard across GPUs).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Workload: the banded config (N=200,000, K=50, off-diagonals iid U[-1,1],
# diagonal = 1.0 x row sum of |off-diagonals|, x_true = 1, b = A x_true,
# P=10, LU_UL, BiCGStab(2) to relative residual 1e-10).
WORKLOAD = dict(name="banded_n200000_k50_d1.0_p10_lu_ul", n=200000, k=50, d=1.0, dist=1, P=10, relTol=1e-10,
                maxit=100)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def oracle_time_to_solution(band, n, k, P, b, relTol, maxit):
    """One setup + solve of the CPU oracle (FP64 preconditioner), seconds."""
    import oracle
    t0 = time.perf_counter()
    pc = oracle.Precond(P, fact=0, dtype="double")
    st = pc.setup_banded(band, n, k)
    x, res = pc.solve(b, band=band, K=k, L=2, maxit=maxit, reltol=relTol)
    dt = time.perf_counter() - t0
    return dt, res, st


def run_reference(args, ws, rank):
    if rank != 0:
        return
    import oracle
    import saplibrary_b200 as sap
    w = WORKLOAD
    band = sap.generate_band_host(w["n"], w["k"], w["d"], w["dist"], seed=1234)
    b = oracle.spmv_banded(band, w["n"], w["k"], np.ones(w["n"]))
    for _ in range(args.warmup):
        oracle_time_to_solution(band, w["n"], w["k"], w["P"], b, w["relTol"], w["maxit"])
    times = []
    res = None
    for _ in range(args.steps):
        dt, res, _ = oracle_time_to_solution(band, w["n"], w["k"], w["P"], b, w["relTol"], w["maxit"])
        times.append(dt)
    t = float(np.mean(times))
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": "time_to_solution", "value": t, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "preconditioner": "fp64", "krylov": "BiCGStab2"},
        "cpu_baseline": {"value": t, "unit": "s", "cores": cores, "kind": "port",
                         "sample": "full workload: setup + BiCGStab(2) solve to rel-res 1e-10 (OpenMP over partitions)"},
        "e2e": {"value": t, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "monitor_code": int(res.code), "iterations": float(res.iterations), "rel_residual": float(res.rel_res_norm),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    ws, rank, local = dist_init()

    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    import saplibrary_b200 as sap

    w = WORKLOAD
    n, k, P = w["n"], w["k"], w["P"]
    seed = 1234 + rank
    band_host = sap.generate_band_host(n, k, w["d"], w["dist"], seed=seed)
    pinned_band = torch.from_numpy(band_host).pin_memory()
    band_np = pinned_band.numpy()
    A = sap.BandedMatrix.from_array(band_np, n, k)
    spmv = sap.MVBanded(A)
    xt = torch.ones(n, device="cuda", dtype=torch.float64)
    b = torch.empty_like(xt)
    spmv(xt, b)
    x = torch.zeros_like(b)
    opts = sap.Options(performReorder=False, variableBandwidth=False, applyScaling=False, factMethod=sap.LU_UL,
                       relTol=w["relTol"], maxNumIterations=w["maxit"])
    solver = sap.Solver(P, opts, prec="double")
    stream = torch.cuda.ExternalStream(solver.stream())

    def step():
        solver.setup(A)
        x.zero_()
        return solver.solve(spmv, b, x)

    for _ in range(max(3, args.warmup)):
        ok = step()
    assert ok, "warm-up solve did not converge"

    # per-kernel breakdown of one step (CUDA events on the launching stream)
    families = ["factor", "transfer", "pass1", "pass2", "pass3", "scan", "reduced_apply", "spmv_banded", "dots"]
    breakdown = {}
    for fam in families:
        sap.profile_select(fam)
        step()
        ms, cnt = sap.profile_read()
        breakdown[fam] = {"ms": ms, "launches": cnt}
    sap.profile_select(None)
    dominant = max(breakdown, key=lambda f: breakdown[f]["ms"])

    # ---- timed region: device events on the solver stream ----------------------
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sap.profile_select(dominant)
    launches0 = sap.kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            ok = step()
        ev1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    gpu_launches = sap.kernel_launch_count() - launches0
    dom_ms, dom_cnt = sap.profile_read()
    sap.profile_select(None)
    ms_total = ev0.elapsed_time(ev1)
    ms_step = ms_total / args.steps
    if ws > 1:
        t = torch.tensor([ms_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    st = solver.getStats()
    code = solver.getMonitorCode()
    err = float(torch.linalg.norm(x - xt) / torch.linalg.norm(xt))

    # ---- end to end through the C ABI with host buffers ---------------------------
    b_host = torch.empty(n, dtype=torch.float64).pin_memory()
    b_host.copy_(b.cpu())
    x_host = torch.zeros(n, dtype=torch.float64).pin_memory()
    b_np, x_np = b_host.numpy(), x_host.numpy()
    solver_h = sap.Solver(P, opts, prec="double")

    def step_e2e():
        Ah = sap.BandedMatrix.from_array(band_np, n, k)   # host -> device copy of the matrix
        solver_h.setup(Ah)
        x_np[:] = 0.0
        ok_ = solver_h.solve(sap.MVBanded(Ah), b_np, x_np)  # b, x0 in; x out
        return ok_

    for _ in range(2):
        step_e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ok_e2e = step_e2e()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if ws > 1:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = band_np.nbytes + 2 * n * 8
    d2h = n * 8

    # ---- roofline of the dominant kernel --------------------------------------------
    peaks, peak_kind = measured_peaks()
    SW = 2 * k + 1
    nfact = 2 * (n - n // P)  # LU rows of partitions 0..P-2 + UL rows of partitions 1..P-1
    bytes_per_launch = {
        "factor": 2 * 8 * SW * nfact,                 # read + write of every factored band column (FP64)
        "pass1": 8 * (k + 1) * n + 8 * n + 8 * n,     # half band + rhs in + F out
        "pass2": 8 * SW * n + 3 * 8 * n,              # full band + F in + Y out
        "pass3": 8 * (k + 1) * n + 2 * 8 * n,         # half band + Y in + out
        "spmv_banded": 8 * SW * n + 16 * n,           # row-major FP64 band + x + y
        "dots": 2 * 8 * n,
        "transfer": 2 * 8 * (k + 1) * n,
        "scan": 0, "reduced_apply": 0,
    }
    avg_ms = dom_ms / max(1, dom_cnt)
    alg = bytes_per_launch.get(dominant, 0)
    achieved = alg / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_source": peak_kind,
                "avg_launch_ms": avg_ms, "launches": dom_cnt}

    line = {
        "metric": "time_to_solution", "value": ms_step / 1e3, "unit": "s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "preconditioner": "fp64 (plain SaP form)", "krylov": "BiCGStab2",
                   "rel_tol": w["relTol"], "parallelism": f"replicas{ws}",
                   "l2": "inputs larger than L2 (FP64 band 161.6 MB)"},
        "solves_per_s": ws * 1e3 / ms_step,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(gpu_launches),
        "roofline": roofline,
        "breakdown_ms": {f: round(v["ms"], 4) for f, v in breakdown.items()},
        "clocks": clk.summary(),
        "monitor_code": code, "iterations": st.numIterations, "rel_residual": st.relResidualNorm,
        "err_vs_xtrue": err, "setup_ms": st.timeSetup, "solve_ms": st.timeSolve,
    }
    if rank == 0 and not args.no_cpu_baseline:
        dt, res, _ = oracle_time_to_solution(band_host, n, k, P, b.cpu().numpy(), w["relTol"], w["maxit"])
        import oracle
        line["cpu_baseline"] = {"value": dt, "unit": "s", "cores": oracle.num_threads(), "kind": "port",
                                "sample": "one full setup + solve of the same workload (FP64 preconditioner)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del solver, solver_h
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
