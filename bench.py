"""Benchmark of the SPIKE-preconditioned Krylov solve on B200.

Workload (one step = one time-to-solution): the 1,000,000-row nonsymmetric
CSR matrix of a 1000 x 1000 2D 5-point convection-diffusion stencil
(diffusion 1, upwinded convection 0.3) plus 2 extra entries per row at
seeded random columns within +-5,000 of the diagonal (values U[-0.1, 0.1]),
rows permuted by a seeded random permutation; b ~ N(0, 1) seeded; P = 16,
drop-off 1e-4; solve to FP64 relative residual 1e-10.  A step is
Solver::setup(A) (DB matching, RCM, drop-off, second-level reordering,
variable band, partition block LU, spike tips, reduced system) followed by
Solver::solve(spmv, b, x) from x = 0 (sap/solver.h:339-562).

Forms timed on it by default: the headline precision form (FP32
preconditioner whose wide-band block products run on the tensor cores in
TF32, FP16 block-scaled sweeps, inside flexible GMRES(50) with FP64
Arnoldi), the same with FP32 sweeps, and the plain FP64 form (FP64
preconditioner, the reference's BiCGStab(2)).  A further form (tf32_refine:
the TF32 preconditioner with FP64 refinement sweeps around BiCGStab(2)) can
be selected with --forms.

Beside it (key "banded"), the banded workloads: N = 2,000,000, K = 200,
N(0,1) off-diagonals, dominance 0.8, P = 32, and the reference's banded
preset N = 200,000, K = 50, U[-1,1], dominance 1.0, P = 10 (both LU_UL,
x_true = ones), each in plain FP64 + BiCGStab(2), TF32 + FGMRES and FP32 +
FGMRES.  cpu_baseline is a complete, measured CPU oracle solve of the 2M-row
banded workload (key "cpu_complete": both banded workloads); the reference
arm (--impl reference) reports itself unavailable, because one complete CPU
solve of the 1M-row sparse workload takes tens of minutes.  Key "ensemble":
128 independent banded systems (N log-uniform in [2e3, 2e5], K in
{8, 16, 32, 64, 128}) solved by one batched call and one by one, each leg
twice, best of the two (--ensemble sets the count, 0 skips it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  With N > 1 (torchrun) every rank solves its
own independent system (replicas; the solve does not shard across GPUs).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="cd2d_m1000_conv0.3_fill2x5000_rowperm_p16_drop1e-4", m=1000, conv=0.3, fill_per_row=2,
                fill_reach=5000, fill_mag=0.1, P=16, drop=1e-4, relTol=1e-10, maxit=100)
FORMS = {
    "tf32_refine": dict(prec="tf32", solver="BiCGStab2", refinementSweeps=6,
                        dtype="f64 Krylov / tf32 factor, f32 sweeps"),
    "tf32_fgmres": dict(prec="tf32", solver="FGMRES", refinementSweeps=0, dtype="f64 Krylov / tf32 factor, f32 sweeps"),
    "tf32f16_fgmres": dict(prec="tf32_f16", solver="FGMRES", refinementSweeps=0,
                           dtype="f64 Krylov / tf32 factor, f16 block-scaled sweeps"),
    "fp64": dict(prec="double", solver="BiCGStab2", refinementSweeps=0, dtype="f64"),
}
HEADLINE = "tf32f16_fgmres"
DEFAULT_FORMS = "tf32f16_fgmres,tf32_fgmres,fp64"
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) over the
# algorithmic bytes of one block-sweep k_tgemv launch, measured with ncu on
# this workload at grid side 310 (block size 3168, the FP32 block size at
# the full size), per bytes of a factor value (4: FP32, 2: FP16 copies); a
# launch's traffic scales with its triangle's bytes
TGEMV_TRAFFIC_RATIO = {4: 1.051, 2: 1.115}


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
        self.out = ""

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
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


def set_grid(m: int) -> None:
    """Grid side of the workload (1000 is the benchmarked size; smaller sides
    serve profiler captures of the same kernels)."""
    if m != WORKLOAD["m"]:
        WORKLOAD["m"] = m
        WORKLOAD["name"] = WORKLOAD["name"].replace("m1000", f"m{m}")


def max_over_ranks(value: float, ws: int) -> float:
    """The maximum of a per-rank value over all ranks (timings are reported
    as max over ranks); the reduction runs on the process group's device."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int) -> int:
    """Every rank solves its own system (replicas): seed of rank r's problem."""
    return 1 + rank


def problems():
    """saplibrary_b200/problems.py loaded by path: the generators need numpy
    only, and importing the package would load the CUDA library (the CPU
    reference arm must not)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_sap_problems", os.path.join(ROOT, "saplibrary_b200", "problems.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_problem(seed: int):
    convection_diffusion_csr = problems().convection_diffusion_csr
    w = WORKLOAD
    rp, ci, v, _ = convection_diffusion_csr(m=w["m"], conv=w["conv"], fill_per_row=w["fill_per_row"],
                                            fill_reach=w["fill_reach"], fill_mag=w["fill_mag"], seed=seed)
    b = np.random.default_rng(seed + 7).standard_normal(w["m"] * w["m"])
    return rp, ci, v, b


# Banded workloads timed beside the headline: the mixed-precision wide band
# (N = 2,000,000, K = 200, N(0,1) off-diagonals, dominance 0.8, P = 32) and
# the reference's banded preset (N = 200,000, K = 50, U[-1,1], dominance 1.0,
# P = 10); both LU_UL on a constant band without reordering, x_true = ones,
# b = A x_true, solved from x = 0 to FP64 relative residual 1e-10.
BANDED = {
    "band_n2000000_k200": dict(n=2_000_000, k=200, d=0.8, dist=2, P=32, seed=1),
    "band_n200000_k50": dict(n=200_000, k=50, d=1.0, dist=1, P=10, seed=1),
}
BANDED_FORMS = {
    "fp64_bicgstab2": dict(prec="double", solver="BiCGStab2"),
    "tf32_fgmres": dict(prec="tf32", solver="FGMRES"),
    "f32_fgmres": dict(prec="float", solver="FGMRES"),
}
# the largest workload whose complete CPU oracle run fits the bench (about a
# minute on 16 host threads); the 1M-row sparse workload takes tens of
# minutes (its FP64 band LU alone runs at ~7 ms per pivot row at K = 3010)
CPU_BASELINE_WORKLOAD = "band_n2000000_k200"
REFERENCE_UNAVAILABLE = (
    "a complete CPU time-to-solution of the 1M-row sparse workload takes tens of minutes per step (the reference "
    "has no CPU preconditioner path; the restated FP64 band LU alone runs at ~7 ms per pivot row at K=3010, ~7 min "
    "for each partition's 62,500 rows), beyond the bench's minutes; complete measured CPU runs of the 2M-row K=200 "
    "and 200k-row K=50 banded workloads are in the GPU arm's cpu_baseline and cpu_complete")


def cpu_complete_banded(name: str, band: np.ndarray):
    """One complete CPU solve of a banded workload by the oracle (the
    reference's algorithm restated, sap/solver.h:339-562 with the banded
    preset of examples/synthetic_banded/driver_banded.cu:166-170): band
    conversion, partition LU/UL, spike tips, reduced system, then
    BiCGStab(2) with the FP64 preconditioner to relative residual 1e-10, on
    all host threads (partitions in parallel).  Nothing is sampled or scaled:
    the value is the measured wall time of the whole solve."""
    import oracle
    c = BANDED[name]
    n, k = c["n"], c["k"]
    b = oracle.spmv_banded(band, n, k, np.ones(n))
    t0 = time.perf_counter()
    pc = oracle.Precond(c["P"], fact=1, dtype="double")
    rc = pc.setup_banded(band, n, k)
    t1 = time.perf_counter()
    if rc != 0:
        raise RuntimeError(f"oracle setup failed on {name}: status {rc}")
    x, res = pc.solve(b, band=band, K=k, L=2, maxit=100, reltol=1e-10)
    t2 = time.perf_counter()
    return {"value": t2 - t0, "unit": "s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"complete solve of {name} (setup {t1 - t0:.2f} s + BiCGStab(2) {t2 - t1:.2f} s, "
                      f"{res.iterations} iterations, relres {res.rel_res_norm:.2e}), FP64 preconditioner, "
                      f"{oracle.num_threads()} host threads",
            "setup_s": t1 - t0, "solve_s": t2 - t1, "iterations": res.iterations, "monitor_code": res.code,
            "rel_residual": res.rel_res_norm, "err_vs_exact": float(np.linalg.norm(x - 1.0) / math.sqrt(n))}, x


def run_reference(args, ws, rank):
    """--impl reference: the CPU path of the reference (restated by the
    oracle) cannot finish one complete solve of this workload within the
    bench, and a sampled-and-scaled time is not a measured time-to-solution,
    so the arm reports itself unavailable with the reason."""
    if rank != 0:
        return
    print(json.dumps({"impl": "reference", "unavailable": REFERENCE_UNAVAILABLE}), flush=True)


def sweep_bytes(bs: int, nb: int, P: int, vbytes: int) -> int:
    """Algorithmic bytes of one block sweep (x <- A_p^-1 x for all partitions):
    the 4*nb-2 triangles of bs(bs+1)/2 factor values it must read (L_ii^-1,
    U_ii^-1, and the off-diagonal factor blocks, whose other triangle is
    structurally zero), the right-hand side and carry vectors read and the
    result written, for P partitions.  vbytes 2: FP16 factor values with FP32
    vectors and one FP32 column scale per factor column."""
    tri = bs * (bs + 1) // 2
    mats = (4 * nb - 2) * tri
    vecs = (4 * nb - 2) * 2 * bs + (2 * nb - 2) * bs
    if vbytes == 2:
        return P * (mats * 2 + vecs * 4 + (4 * nb - 2) * bs * 4)
    return P * (mats + vecs) * vbytes


def time_banded(sap, torch, name: str, warm: int, steps: int, ws: int) -> dict:
    """GPU time-to-solution of every banded form on one banded workload:
    one step = Solver::setup(A) + solve(spmv, b, x) from x = 0, timed with
    CUDA events on the solver stream after each step; tts_s is the median
    step (the host side of a step on a shared machine shows occasional
    stalls of 0.1-2 s), tts_mean_s the mean, step_ms every step.  Also the
    error against the exact
    solution (ones) and the FP64 form's solution (key _x, for the comparison
    with the CPU oracle's)."""
    c = BANDED[name]
    n, k = c["n"], c["k"]
    A = sap.BandedMatrix(n, k, c["d"], dist=c["dist"], seed=c["seed"])
    spmv = sap.MVBanded(A)
    ones = torch.ones(n, dtype=torch.float64, device="cuda")
    b = torch.empty_like(ones)
    spmv(ones, b)
    x = torch.zeros_like(b)
    out = {"n": n, "K": k, "P": c["P"], "dominance": c["d"], "values": "N(0,1)" if c["dist"] == 2 else "U[-1,1]"}
    for form, f in BANDED_FORMS.items():
        opts = sap.Options(solverType=getattr(sap, f["solver"]), performReorder=False, variableBandwidth=False,
                           applyScaling=False, factMethod=sap.LU_UL, relTol=1e-10, maxNumIterations=400)
        solver = sap.Solver(c["P"], opts, prec=f["prec"])
        stream = torch.cuda.ExternalStream(solver.stream())

        def step():
            solver.setup(A)
            x.zero_()
            return solver.solve(spmv, b, x)

        ok = all([step() for _ in range(warm)])
        torch.cuda.synchronize()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        evs[0].record(stream)
        for i in range(steps):
            ok = step() and ok
            evs[i + 1].record(stream)
        torch.cuda.synchronize()
        step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
        st = solver.getStats()
        r = torch.empty_like(b)
        spmv(x, r)
        med = sorted(step_ms)[steps // 2]
        out[form] = {"tts_s": max_over_ranks(med / 1e3, ws), "tts_mean_s": max_over_ranks(sum(step_ms) / steps / 1e3, ws),
                     "steps": steps, "ok": bool(ok), "step_ms": [round(t, 2) for t in step_ms],
                     "monitor_code": solver.getMonitorCode(), "iterations": st.numIterations,
                     "true_rel_residual": float(torch.linalg.norm(b - r) / torch.linalg.norm(b)),
                     "err_vs_exact": float(torch.linalg.norm(x - ones) / math.sqrt(n)),
                     "setup_ms": round(st.timeSetup, 2), "solve_ms": round(st.timeSolve, 2),
                     "block_size": solver.blockLayout()[0]}
        if form == "fp64_bicgstab2":
            out["_x"] = x.cpu().numpy().copy()
        del solver, stream
        torch.cuda.empty_cache()
    if "fp64_bicgstab2" in out:
        base = out["fp64_bicgstab2"]["tts_s"]
        out["speedup_vs_plain_fp64"] = {f: base / out[f]["tts_s"] for f in BANDED_FORMS if f in out}
    del A, spmv
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--forms", default=DEFAULT_FORMS, help="comma-separated forms to time (" + ", ".join(FORMS) + ")")
    ap.add_argument("--m", type=int, default=WORKLOAD["m"], help="grid side (profiler captures only)")
    ap.add_argument("--ensemble", type=int, default=128,
                    help="systems of the batched-ensemble comparison (0: skip)")
    ap.add_argument("--banded", default=",".join(BANDED),
                    help="banded workloads timed beside the headline (" + ", ".join(BANDED) + "; empty: none)")
    args = ap.parse_args()
    set_grid(args.m)
    ws, rank, local = dist_init()

    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    import saplibrary_b200 as sap

    w = WORKLOAD
    warm = max(3, args.warmup)
    rp, ci, v, b_np = make_problem(seed=rank_seed(rank))
    n = len(rp) - 1
    A = sap.CsrMatrix(rp, ci, v)
    spmv = sap.SpmvCusp(A)
    b = torch.tensor(b_np, device="cuda")
    x = torch.zeros_like(b)

    def solver_for(form):
        f = FORMS[form]
        opts = sap.Options(solverType=getattr(sap, f["solver"]), dropOffFraction=w["drop"], relTol=w["relTol"],
                           maxNumIterations=w["maxit"] if f["solver"] != "FGMRES" else 4 * w["maxit"],
                           refinementSweeps=f["refinementSweeps"])
        return sap.Solver(w["P"], opts, prec=f["prec"])

    results = {}
    forms = [f for f in args.forms.split(",") if f]
    if HEADLINE not in forms:
        forms.insert(0, HEADLINE)
    peaks, peak_kind = measured_peaks()
    clocks, head_launches = None, 0
    for form in forms:
        solver = solver_for(form)
        stream = torch.cuda.ExternalStream(solver.stream())

        def step():
            solver.setup(A)
            x.zero_()
            return solver.solve(spmv, b, x)

        ok = False
        for _ in range(warm):
            ok = step()
        assert ok, f"{form}: warm-up solve did not converge"
        steps = args.steps if form == HEADLINE else min(args.steps, 3)
        # ---- timed region: device events on the solver stream ----------------
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sap.profile_select("block_sweep")
        launches0, lib0 = sap.kernel_launch_count(), sap.library_call_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            for _ in range(steps):
                ok = step()
            ev1.record(stream)
            torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        sweep_ms, sweep_cnt = sap.profile_read()
        sap.profile_select(None)
        launches = sap.kernel_launch_count() - launches0
        lib_calls = sap.library_call_count() - lib0
        ms_step = max_over_ranks(ev0.elapsed_time(ev1) / steps, ws)
        st = solver.getStats()
        bs, nb, vb = solver.blockLayout()
        _, K, P = solver.info()
        # true FP64 residual of the last step's solution
        r = torch.empty_like(b)
        spmv(x, r)
        true_rel = float(torch.linalg.norm(b - r) / torch.linalg.norm(b))
        res = {
            "tts_s": ms_step / 1e3, "steps": steps, "ok": bool(ok), "monitor_code": solver.getMonitorCode(),
            "iterations": st.numIterations, "rel_residual": st.relResidualNorm, "true_rel_residual": true_rel,
            "K": K, "P": P, "block_size": bs, "blocks_per_partition": nb, "value_bytes": vb,
            "gpu_launches_per_step": launches / steps, "cublas_calls_per_step": lib_calls / steps,
            "stage_ms": {k: round(getattr(st, k), 2) for k in
                         ("time_DB", "time_reorder", "time_dropOff", "time_cpu_assemble", "time_transfer",
                          "time_bandLU", "time_assembly", "time_fullLU", "timeSetup", "timeSolve")},
        }
        if bs > 0 and sweep_cnt > 0:
            avg = sweep_ms / sweep_cnt
            alg = sweep_bytes(bs, nb, P, vb)
            res["block_sweep"] = {"avg_ms": avg, "launches": sweep_cnt, "bytes": alg,
                                  "gbs": alg / (avg * 1e-3) / 1e9}
        results[form] = res
        if form == HEADLINE:
            clocks = clk.summary()
            head_launches = launches
        del solver, stream
        torch.cuda.empty_cache()

    head = results[HEADLINE]

    # ---- SpMV of the Krylov loop (k_spmv_csr_blocks) against HBM: y = A x,
    # the L2 flushed before every launch (a 256 MB write, then a 256 MB read
    # that leaves clean lines), the kernel timed by the library's CUDA events
    # on its launching stream ----------------------------------------------------
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    clean = torch.ones(64 << 20, dtype=torch.float32, device="cuda")
    y_sp = torch.empty_like(b)
    spmv(b, y_sp)
    sp_times = []
    for _ in range(10):
        flush.fill_(1.0)
        clean.sum()
        torch.cuda.synchronize()
        sap.profile_select("spmv_csr")
        spmv(b, y_sp)
        ms, cnt = sap.profile_read()
        sap.profile_select(None)
        sp_times.append(ms / max(cnt, 1))
    sp_bytes = 12 * int(rp[-1]) + 4 * (n + 1) + 16 * n  # values + column indices, row offsets, x, y
    sp_best = min(sp_times)
    spmv_roof = {"kernel": "k_spmv_csr_blocks", "bound": "hbm", "achieved": sp_bytes / sp_best / 1e6, "unit": "GB/s",
                 "peak": peaks["hbm_gbs"], "frac": sp_bytes / sp_best / 1e6 / peaks["hbm_gbs"], "bytes": sp_bytes,
                 "best_ms": sp_best, "peak_source": peak_kind}
    del flush, clean, y_sp

    # ---- end to end through the public API with host buffers ----------------------
    e2e = None
    if not args.no_e2e:
        solver_h = solver_for(HEADLINE)
        b_host = torch.from_numpy(b_np.copy()).pin_memory()
        x_host = torch.zeros(n, dtype=torch.float64).pin_memory()
        bh, xh = b_host.numpy(), x_host.numpy()

        def step_e2e():
            Ah = sap.CsrMatrix(rp, ci, v)  # host -> device copy of the matrix
            solver_h.setup(Ah)
            xh[:] = 0.0
            return solver_h.solve(sap.SpmvCusp(Ah), bh, xh)  # b, x0 in; x out

        for _ in range(2):
            step_e2e()
        torch.cuda.synchronize()
        # every step timed on its own (the result is on the host when a step
        # returns): the median is the value, the mean is reported beside it
        # (host stalls of a shared machine land in single steps)
        e2e_steps = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            step_e2e()
            e2e_steps.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(sorted(e2e_steps)[len(e2e_steps) // 2], ws)
        h2d = rp.nbytes + ci.nbytes + v.nbytes + 2 * n * 8
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": n * 8,
               "mean_s": max_over_ranks(sum(e2e_steps) / len(e2e_steps), ws),
               "step_s": [round(t, 4) for t in e2e_steps]}
        del solver_h

    # ---- roofline of the dominant kernel: the block-sweep gemv (k_tgemv) ----------
    roofline = None
    if "block_sweep" in head:
        bsw = head["block_sweep"]
        ratio = TGEMV_TRAFFIC_RATIO.get(head["value_bytes"])
        kern = ("k_sweep<float, 8, __half> (one cooperative launch per block sweep)" if head["value_bytes"] == 2
                else "k_tgemv (one block sweep = 4*nb-2 launches)")
        roofline = {"kernel": kern, "bound": "hbm", "achieved": bsw["gbs"],
                    "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": bsw["gbs"] / peaks["hbm_gbs"],
                    "traffic": int(ratio * bsw["bytes"]) if ratio else None,
                    "traffic_source": "ncu ratio of one block-sweep launch at grid side 310, scaled" if ratio else None,
                    "peak_source": peak_kind, "avg_sweep_ms": bsw["avg_ms"], "bytes_per_sweep": bsw["bytes"]}

    line = {
        "metric": "time_to_solution", "value": head["tts_s"], "unit": "s", "n_gpus": ws, "steps": args.steps,
        "warmup": warm, "ms_per_step": head["tts_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": FORMS[HEADLINE]["dtype"], "data": "synthetic",
        "config": {"workload": w["name"], "form": HEADLINE, "krylov": "flexible GMRES(50), FP64 Arnoldi",
                   "rel_tol": w["relTol"], "parallelism": f"replicas{ws}",
                   "l2": "inputs larger than L2 (CSR 84 MB, factors tens of GB)"},
        "solves_per_s": ws / head["tts_s"],
        "plain_fp64_tts_s": results["fp64"]["tts_s"] if "fp64" in results else None,
        "speedup_vs_plain_fp64": (results["fp64"]["tts_s"] / head["tts_s"]) if "fp64" in results else None,
        "e2e": e2e,
        "gpu_launches": int(head_launches),
        "roofline": roofline,
        "spmv_roofline": spmv_roof,
        "clocks": clocks,
        "forms": results,
    }
    # ---- banded workloads: GPU forms, then the complete CPU oracle runs ----------
    banded = [b for b in args.banded.split(",") if b]
    if banded:
        # at least 9 timed steps, 15 for the 200k-row preset (~20 ms a step):
        # host stalls on a shared machine come in clusters that can reach
        # the median of fewer steps
        line["banded"] = {name: time_banded(sap, torch, name, warm, max(args.steps, 9 if BANDED[name]["n"] >= 10**6 else 15),
                                            ws) for name in banded}
    if args.ensemble > 0:
        # batched ensemble of independent banded systems (N log-uniform in
        # [2e3, 2e5], K in {8..128}, FP32 preconditioner, FGMRES to 1e-10):
        # one solve_batch call against the same systems solved one by one
        from saplibrary_b200 import ensemble
        line["ensemble"] = ensemble.run(count=args.ensemble, seed=3, P=8, prec="float", reps=2)
    if rank == 0 and not args.no_cpu_baseline:
        cpu_runs = {}
        for name in banded:
            c = BANDED[name]
            band = sap.generate_band_host(c["n"], c["k"], c["d"], c["dist"], seed=c["seed"])
            run, xo = cpu_complete_banded(name, band)
            del band
            gx = line["banded"][name].get("_x")
            if gx is not None:
                run["gpu_fp64_x_vs_cpu_x"] = float(np.linalg.norm(gx - xo) / np.linalg.norm(xo))
            cpu_runs[name] = run
        if CPU_BASELINE_WORKLOAD in cpu_runs:
            line["cpu_baseline"] = dict(cpu_runs[CPU_BASELINE_WORKLOAD], workload=CPU_BASELINE_WORKLOAD)
        line["cpu_complete"] = cpu_runs
    for name in banded:
        line["banded"][name].pop("_x", None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
