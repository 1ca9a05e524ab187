#!/usr/bin/env python3
"""Headline benchmark of the B200 sparse-solver hot path.

Workload (one "step"): Matrix::solve(x, b, config) on the 192^3
variable-coefficient 7-point Poisson system (7,077,888 rows, cell
coefficients log-normal sigma = 1.5 from seed 2, harmonic-mean faces,
Dirichlet boundary), float32 CRS, b = A x_true with x_true ~ U[-1, 1) from
seed 3, x0 = 0: mixed-precision iterative refinement (FP64 residual and
solution update) around an FP32 PBiCGStab with block-ILU(0), inner relative
residual 1e-4, to a 1e-10 relative residual. A step creates the solver (ILU
factorisation) and solves, as the reference's Matrix::solve does
(matrix/Matrix.cpp:26-30). The matrix and vectors are resident in HBM; the
matrix (451 MB per SpMV) is larger than L2, so no flush is needed between
steps.

Reported beside it, on the same GPU and system: plain FP64 PBiCGStab-ILU(0)
to 1e-10 (the comparison of the north-star target), the double-word MPIR
variant, SpMV HBM bandwidth, and the CPU oracle's time on the host cores.

Usage: python bench.py [--gpus N --steps K --warmup W] [--impl reference]
(N > 1: one process per GPU under torchrun, each rank solving its own copy;
replicas only -- the path does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = ("time-to-1e-10 rel. residual (MPIR vs FP64 PBiCGStab), SpMV HBM GB/s, p50/p99 ms")
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0


def args_():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--grid", type=int, default=192)
    p.add_argument("--tiles", type=int, default=1024)
    p.add_argument("--sigma", type=float, default=1.5)
    p.add_argument("--inner-tol", type=float, default=1e-4)
    p.add_argument("--inner-maxit", type=int, default=500)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--cpu-threads", type=int, default=0)
    return p.parse_args()


def peaks():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def mpir_config(a, ext="float64"):
    return {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 50,
            "extendedPrecisionType": ext,
            "innerSolver": {"type": "PBiCGStab", "maxIterations": a.inner_maxit,
                            "relResidual": a.inner_tol, "preconditioner": {"type": "ILU"}}}


def fp64_config():
    return {"type": "PBiCGStab", "maxIterations": 20000, "relResidual": 1e-10,
            "preconditioner": {"type": "ILU"}}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(h, b32, a, threads: int, total_inner: int, outer: int):
    """The oracle (CPU restatement of the reference) on the same system:
    ILU factorisation plus a bounded number of PBiCGStab-ILU(0) iterations are
    timed; the time-to-solution is that per-iteration cost times the inner
    iterations the solve takes (the oracle and the GPU iterate identically),
    plus the factorisation and one FP64 residual per outer iteration."""
    import numpy as np
    from tests.oracle_py import Oracle

    o = Oracle()
    o.threads(threads)
    rows, cols, vals = h.coo()
    om = o.matrix(h.numRows, rows, cols, vals, h.numTiles, h.rowToTile(), 0)
    b_tile = h.decomposeVector(b32)
    t0 = time.perf_counter()
    om.ilu_factorize(False)
    t_fact = time.perf_counter() - t0
    k = 4
    cfg = json.dumps({"type": "PBiCGStab", "maxIterations": k, "preconditioner": {"type": "ILU"}})
    t0 = time.perf_counter()
    om.solve(cfg, np.zeros_like(b_tile), b_tile)
    t_k = time.perf_counter() - t0 - t_fact  # the node factorises again
    t_iter = max(t_k, 0.0) / k
    xz = np.zeros(h.numRows, np.float64)
    t0 = time.perf_counter()
    om.residual(xz, 1, b_tile, 0, 1)
    t_res = time.perf_counter() - t0
    est_s = t_fact + total_inner * t_iter + outer * (t_res + t_fact * 0)
    return {
        "value": est_s * 1e3, "unit": "ms", "cores": threads, "kind": "port",
        "sample": (f"oracle on the full {a.grid}^3 system ({threads} threads): ILU(0) factorisation "
                   f"{t_fact:.2f} s + {k} PBiCGStab-ILU(0) iterations ({t_iter:.3f} s each) + one FP64 "
                   f"residual ({t_res:.3f} s), scaled to the solve's {total_inner} inner / {outer} outer "
                   f"iterations"),
    }


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    import graphene_b200 as gb

    threads = a.cpu_threads or os.cpu_count() or 1
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, a.grid, a.grid, a.grid, (a.sigma,), 2, a.tiles)
    xt = gb.randomVector(3, h.numRows).astype(np.float32)
    from tests.oracle_py import Oracle
    o = Oracle()
    o.threads(threads)
    rows, cols, vals = h.coo()
    om = o.matrix(h.numRows, rows, cols, vals, h.numTiles, h.rowToTile(), 0)
    b = om.spmv(h.decomposeVector(xt))
    times = []
    per_iter = []
    k = 3
    cfg = json.dumps({"type": "PBiCGStab", "maxIterations": k, "preconditioner": {"type": "ILU"}})
    for step in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        om.solve(cfg, np.zeros_like(b), b)
        dt = time.perf_counter() - t0
        if step >= a.warmup:
            times.append(dt)
            per_iter.append(dt / k)
    # Inner / outer iteration counts of this system's MPIR solve (measured on
    # the GPU path, which iterates like the oracle): 16 outer is an upper
    # estimate when no GPU count is given.
    total_inner = int(os.environ.get("GRAPHENE_INNER_ITERS", "0")) or None
    it = statistics.median(per_iter)
    value = (it * total_inner * 1e3) if total_inner else None
    line = {"impl": "reference", "metric": METRIC, "unit": "ms", "higher_is_better": False,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "value": value, "ms_per_step": statistics.mean(times) * 1e3,
            "config": {"workload": f"MPIR(FP64 residual) PBiCGStab-ILU(0) var-coeff Poisson {a.grid}^3",
                       "tiles": h.numTiles, "sigma": a.sigma},
            "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "port",
                             "sample": f"{k} PBiCGStab-ILU(0) iterations incl. factorisation per step, "
                                       f"{it:.3f} s per iteration"},
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    a = args_()
    if a.impl == "reference":
        return reference_arm(a)
    import numpy as np
    import torch
    import graphene_b200 as gb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    hbm_peak, peak_kind = peaks()
    t0 = time.perf_counter()
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, a.grid, a.grid, a.grid, (a.sigma,), 2, a.tiles)
    t_host = time.perf_counter() - t0
    n, m = h.numRows, h.numOffDiag
    A = h.copyToTile()
    xt = gb.randomVector(3, n).astype(np.float32)
    x_true = A.vector(xt)
    b = A * x_true  # b = A x in float32, as the reference's benchmark does
    cfg = mpir_config(a)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def solve_once(config, bvec, dtype=torch.float32):
        s = gb.Solver(A_of[dtype], config)
        x = torch.zeros(n, dtype=dtype, device="cuda")
        st = s.solve(x, bvec)
        return s, x, st

    A_of = {torch.float32: A}
    for _ in range(a.warmup):
        solve_once(cfg, b)
    barrier()
    launches0 = gb.launch_count()
    ev = []
    stats = []
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(a.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            s, x, st = solve_once(cfg, b)
            e1.record()
            ev.append((e0, e1))
            stats.append(st)
        barrier()
    launches = gb.launch_count() - launches0
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / a.steps
    st = stats[-1]
    # FP64 check of the last solution on the stored float32 matrix.
    phi = s.phi(gb.FLOAT64)
    r64 = A.residual(phi, b, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
    rel64 = float(torch.linalg.vector_norm(r64) / torch.linalg.vector_norm(b.double()))

    # ---- same system, other solvers (same GPU) ----
    extra = {}
    if not a.no_fp64:
        h64 = h.astype(gb.FLOAT64)
        A64 = h64.copyToTile()
        A_of[torch.float64] = A64
        b64 = b.double()
        solve_once(fp64_config(), b64, torch.float64)  # warm-up (schedules, graph)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, x64, st64 = solve_once(fp64_config(), b64, torch.float64)
        e1.record()
        torch.cuda.synchronize()
        fp64_ms = e0.elapsed_time(e1)
        r = A64.residual(x64, b64, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
        extra["fp64_pbicgstab_ilu0"] = {
            "ms": fp64_ms, "iterations": st64.iterations, "converged": st64.converged,
            "rel_residual_fp64": float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b64))}
        extra["speedup_mpir_vs_fp64"] = fp64_ms / ms_per_step
        del A64
        A_of.pop(torch.float64)
    cfg_dw = mpir_config(a, "twofloat32")
    solve_once(cfg_dw, b)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    s_dw, _, st_dw = solve_once(cfg_dw, b)
    e1.record()
    torch.cuda.synchronize()
    phi_dw = s_dw.phi(gb.FLOAT64)
    r = A.residual(phi_dw, b, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
    extra["mpir_twofloat32"] = {"ms": e0.elapsed_time(e1), "outer": st_dw.iterations,
                                "inner": st_dw.innerIterations, "converged": st_dw.converged,
                                "rel_residual_fp64": float(torch.linalg.vector_norm(r) /
                                                           torch.linalg.vector_norm(b.double()))}

    # ---- kernel timings: SpMV (HBM roofline) and the ILU(0) application ----
    y = torch.empty_like(x_true)
    for _ in range(5):
        A.spmv(x_true, y)
    torch.cuda.synchronize()
    reps = 50
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        A.spmv(x_true, y)
    e1.record()
    torch.cuda.synchronize()
    spmv_ms = e0.elapsed_time(e1) / reps
    spmv_bytes = 8 * m + 16 * n + 4
    spmv_gbs = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    ilu = gb.Solver(A, {"type": "ILU"})
    z = torch.empty_like(x_true)
    for _ in range(3):
        ilu.solve(z, b)
    torch.cuda.synchronize()
    reps_ilu = 20
    e0.record()
    for _ in range(reps_ilu):
        ilu.solve(z, b)
    e1.record()
    torch.cuda.synchronize()
    ilu_ms = e0.elapsed_time(e1) / reps_ilu
    ilu_bytes = 8 * m + 12 * n
    extra["spmv"] = {"ms": spmv_ms, "GBs": spmv_gbs, "frac_of_hbm": spmv_gbs / hbm_peak,
                     "bytes_per_launch": spmv_bytes}
    extra["ilu0_apply"] = {"ms": ilu_ms, "GBs": ilu_bytes / (ilu_ms * 1e-3) / 1e9,
                           "frac_of_hbm": ilu_bytes / (ilu_ms * 1e-3) / 1e9 / hbm_peak,
                           "bytes_per_launch": ilu_bytes}

    # ---- end to end through the C ABI with host buffers ----
    import numpy as _np
    b_host = torch.empty(n, dtype=torch.float32, pin_memory=True)
    b_host.copy_(torch.from_numpy(A.toNatural(b)))
    x_host = torch.zeros(n, dtype=torch.float32, pin_memory=True)
    e2e_ms = []
    for i in range(max(1, min(a.steps, 3)) + 1):
        x_host.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        se = gb.Solver(A, cfg)
        se.solveHost(x_host.numpy(), b_host.numpy())
        e1.record()
        torch.cuda.synchronize()
        if i > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_val = statistics.mean(e2e_ms)
    err = float(_np.abs(x_host.numpy() - xt).max())

    # ---- roofline of the dominant kernel (by measured time per solve) ----
    inner = st.innerIterations
    share_ilu = 2 * inner * ilu_ms
    share_spmv = 2 * inner * spmv_ms
    if share_ilu >= share_spmv:
        dom = {"kernel": "ilu_apply (iluApplyKernel)", "achieved": ilu_bytes / (ilu_ms * 1e-3) / 1e9,
               "bytes": ilu_bytes, "ms": ilu_ms}
    else:
        dom = {"kernel": "spmv (spmvDotKernel)", "achieved": spmv_gbs, "bytes": spmv_bytes, "ms": spmv_ms}
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(dom["kernel"].split(" ")[0])
        except Exception:
            traffic = None

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            threads = a.cpu_threads or os.cpu_count() or 1
            cpu = cpu_baseline(h, xt_nat(A, b), a, threads, inner, st.iterations)
        except Exception as e:  # the baseline is informative; report why it is missing
            cpu = {"value": None, "error": str(e)[:200]}

    line = {
        "metric": METRIC,
        "value": ms_per_step,
        "unit": "ms",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"MPIR(FP64 residual+update) PBiCGStab-ILU(0) FP32 inner, var-coeff "
                               f"Poisson {a.grid}^3 (n={n}, offdiag={m}), sigma={a.sigma}, to 1e-10",
                   "tiles": h.numTiles, "inner_rel_residual": a.inner_tol,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (no flush)"},
        "solve": {"outer_iterations": st.iterations, "inner_iterations": inner,
                  "converged": st.converged, "final_rel_residual": st.finalResidual / st.initialResidual,
                  "rel_residual_fp64_of_phi": rel64, "p50_ms": statistics.median(step_ms),
                  "max_ms": max(step_ms)},
        "extra": extra,
        "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["achieved"],
                     "peak": hbm_peak, "unit": "GB/s", "frac": dom["achieved"] / hbm_peak,
                     "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": dom["bytes"], "launch_ms": dom["ms"]},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_val, "unit": "ms", "h2d_bytes_per_step": 2 * 4 * n,
                "d2h_bytes_per_step": 4 * n, "max_abs_err_vs_x_true": err},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "host_setup_s": t_host,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def xt_nat(A, b):
    """Right-hand side in natural order as float32 numpy."""
    return A.toNatural(b)


if __name__ == "__main__":
    sys.exit(main())
