#!/usr/bin/env python3
"""Headline benchmark of the B200 sparse-solver hot path.

Workload (one "step"): Matrix::solve(x, b, config) on the 192^3
variable-coefficient 7-point Poisson system (7,077,888 rows, 42,246,144
off-diagonals; cell coefficients log-normal sigma = 1.5 from seed 2,
harmonic-mean faces, Dirichlet boundary), float32 CRS in 2368 tiles (16 per
SM of the B200's 148: two full waves of the substitution kernel),
b = A x_true with x_true ~ U[-1, 1) from seed 3, x0 = 0: mixed-precision
iterative refinement (FP64 residual and solution update) around an FP32
PBiCGStab with block-ILU(0), inner relative residual 1e-4, to a 1e-10
relative residual. A step creates the solver (ILU factorisation) and
solves, as the reference's Matrix::solve does (matrix/Matrix.cpp:26-30).
Matrix and vectors are resident in HBM; the matrix (451 MB per SpMV) is
larger than L2, so no flush is needed between steps.

Reported beside it on the same GPU and system: plain FP64 PBiCGStab-ILU(0)
to 1e-10 (the north-star comparison), MPIR with a double-word residual and
with inner tolerance 1e-3, SpMV and ILU(0) HBM bandwidth, the end-to-end
call with host buffers, and the CPU oracle's time on the host cores.

--impl reference: the CPU oracle (the reference algorithm restated in C++;
the reference itself needs the Poplar SDK) on all host cores, same system
and solver: one full MPIR solve (measured) and bounded per-step samples.

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

METRIC = "time-to-1e-10 rel. residual (MPIR vs FP64 PBiCGStab), SpMV HBM GB/s, p50/p99 ms"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0
SEED_MATRIX, SEED_X = 2, 3
# Tiles of the 192^3 system: 16 per SM on 148 SMs. The ILU(0) substitution
# keeps 8 tiles resident per SM, so 2368 tiles run in two full waves; on
# B200 MPIR took 126.6 ms at 2368 tiles against 144.5 ms at 2048 and FP64
# PBiCGStab 167.5 ms against 172.8 ms (block-ILU(0) over these tiles needs
# 273 inner iterations against 327).
C3_TILES = 2368


def max_over_ranks(value, dist=None, device="cuda"):
    """The largest `value` over the ranks of the process group, for timing a
    multi-GPU run as its slowest rank (`value` itself without a group)."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--grid", type=int, default=192)
    p.add_argument("--tiles", type=int, default=C3_TILES)
    p.add_argument("--sigma", type=float, default=1.5)
    p.add_argument("--inner-tol", type=float, default=1e-4)
    p.add_argument("--inner-maxit", type=int, default=500)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true")
    p.add_argument("--tiles-per-block", type=int, default=0,
                   help="ILU ring: tiles a block (0: automatic; 2 also sets four compute warps), for profiling "
                        "the grouped kernel on a case where it is not chosen automatically")
    p.add_argument("--cpu-threads", type=int, default=0)
    p.add_argument("--case", choices=sorted(CASES), default=None,
                   help="run one benchmark configuration alone (timing and profiling): "
                        "W untimed + K timed solves of it, one JSON line")
    return p.parse_args()


def hbm_peak():
    try:
        return float(json.loads(PEAKS_FILE.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def mpir_config(a, ext="float64", tol=None):
    pre = {"type": "ILU"}
    if a.tiles_per_block > 0:
        pre.update({"tilesPerBlock": a.tiles_per_block, "computeWarps": 4 if a.tiles_per_block > 1 else 0})
    return {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 50,
            "extendedPrecisionType": ext,
            "innerSolver": {"type": "PBiCGStab", "maxIterations": a.inner_maxit,
                            "relResidual": a.inner_tol if tol is None else tol,
                            "preconditioner": pre}}


FP64_CONFIG = {"type": "PBiCGStab", "maxIterations": 20000, "relResidual": 1e-10,
               "preconditioner": {"type": "ILU"}}


def workload_name(a, n, m):
    return (f"MPIR(FP64 residual+update) over FP32 PBiCGStab-ILU(0), var-coeff 7-pt Poisson "
            f"{a.grid}^3 (n={n}, offdiag={m}), sigma={a.sigma}, {a.tiles} tiles, to 1e-10")


def bench_config(a, world):
    """The `config` of both arms' JSON lines (identical by construction)."""
    g = a.grid
    n, m = g ** 3, 6 * g * g * (g - 1)  # 7-point stencil: 2 x 3 (g - 1) g^2 off-diagonals
    return {"workload": workload_name(a, n, m), "tiles": a.tiles, "inner_rel_residual": a.inner_tol,
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (no flush)"}


class ClockSampler:
    """nvidia-smi clock / throttle samples; summary over a marked window."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []
        self.window = (0, None)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def mark_start(self):
        self.window = (len(self.lines), None)

    def mark_end(self):
        time.sleep(0.25)
        self.window = (self.window[0], len(self.lines))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        lo, hi = self.window
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[lo:hi]:
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


def oracle_system(a, threads):
    """The headline system built by the oracle alone (its own generator,
    coordinate bisection and seeded vectors; no part of the product
    library): (oracle matrix, b in tile order, float32)."""
    import numpy as np
    from tests.oracle_py import Oracle

    o = Oracle()
    o.threads(threads)
    om = o.grid_system(1, a.grid, a.grid, a.grid, (a.sigma,), SEED_MATRIX, a.tiles)
    xt = o.random_vector(SEED_X, om.n).astype(np.float32)
    return om, om.spmv(om.decompose(xt))


def oracle_sample(om, b_tile, k=3):
    """Times the oracle's ILU(0) factorisation, a PBiCGStab-ILU(0) solve of
    one iteration and one of 1 + k iterations, and one FP64 residual.
    Returns (t_fact, t_iter, t_res, t_setup): the per-iteration time is the
    difference of the two solves over k (their factorisation and set-up
    cancel), t_setup a solve's cost besides its factorisation and
    iterations."""
    import numpy as np

    t0 = time.perf_counter()
    om.ilu_factorize(False)
    t_fact = time.perf_counter() - t0
    times = []
    for its in (1, 1 + k):
        cfg = json.dumps({"type": "PBiCGStab", "maxIterations": its, "preconditioner": {"type": "ILU"}})
        t0 = time.perf_counter()
        om.solve(cfg, np.zeros_like(b_tile), b_tile)
        times.append(time.perf_counter() - t0)
    t_iter = max(times[1] - times[0], 0.0) / k
    t_setup = max(times[0] - t_fact - t_iter, 0.0)  # each solve factorises once more
    t0 = time.perf_counter()
    om.residual(np.zeros(len(b_tile)), 1, b_tile, 0, 1)
    t_res = time.perf_counter() - t0
    return t_fact, t_iter, t_res, t_setup


def project_ms(sample, outer, inner):
    """An MPIR solve's time from an oracle sample: one factorisation, per
    outer step a residual and an inner solve's set-up, the inner
    iterations."""
    t_fact, t_iter, t_res, t_setup = sample
    return (t_fact + outer * (t_res + t_setup) + inner * t_iter) * 1e3


def reference_arm(a):
    """The CPU oracle on the host cores (rank 0 only). Everything it runs is
    the oracle's: the system (generator, bisection, seeded x_true, b = A x in
    FP32) and the MPIR solve. One full solve is measured for the iteration
    counts and as a check; each of the W + K steps is a bounded sample of
    the same solve (ILU(0) factorisation, 3 PBiCGStab-ILU(0) iterations, one
    FP64 residual), and `value` scales the timed steps' median sample to the
    full solve's iteration counts."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    import numpy as np

    threads = a.cpu_threads or os.cpu_count() or 1
    om, b = oracle_system(a, threads)
    t0 = time.perf_counter()
    _, st, _, _ = om.solve(json.dumps(mpir_config(a)), np.zeros_like(b), b)
    full_ms = (time.perf_counter() - t0) * 1e3
    samples, step_ms = [], []
    for step in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        s = oracle_sample(om, b)
        if step >= a.warmup:
            samples.append(s)
            step_ms.append((time.perf_counter() - t0) * 1e3)
    med = tuple(statistics.median(x[i] for x in samples) for i in range(4))
    t_fact, t_iter, t_res, t_setup = med
    value = project_ms(med, st.iterations, st.inner_iterations)
    sample = (f"each step: ILU(0) factorisation, PBiCGStab-ILU(0) solves of 1 and 4 iterations and one FP64 "
              f"residual of the oracle on the full system, {threads} threads ({t_fact:.2f} s, "
              f"{t_iter:.3f} s/iteration, {t_res:.3f} s, solve set-up {t_setup:.3f} s); value = those medians "
              f"scaled to the full solve's {st.iterations} outer / {st.inner_iterations} inner iterations; one "
              f"full solve measured {full_ms:.0f} ms (converged={bool(st.converged)})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "ms",
            "higher_is_better": False, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": statistics.mean(step_ms), "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 outer", "data": "synthetic (seeded generator)",
            "config": bench_config(a, int(os.environ.get("WORLD_SIZE", "1"))),
            "full_solve_ms": full_ms, "outer_iterations": st.iterations,
            "inner_iterations": st.inner_iterations,
            "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def pbicgstab(precond, tol, maxit=1000):
    pre = {"ILU": {"type": "ILU"},
           "GS": {"type": "GaussSeidel", "numSweeps": 2, "numFixedIterations": 2}}[precond]
    return {"type": "PBiCGStab", "maxIterations": maxit, "relResidual": tol, "preconditioner": pre}


def timed_solve(gb, A, cfg, b, reps=2):
    """Best of `reps` (solver creation + solve) by CUDA events, after one
    warm-up; returns (ms, stats, relative FP64 residual of x)."""
    import torch
    n = A.numRows

    def once():
        x = torch.zeros(n, dtype=b.dtype, device="cuda")
        s = gb.Solver(A, cfg)
        st = s.solve(x, b)
        return x, st, s
    once()
    best = None
    x = st = s = None
    for _ in range(reps):
        x = s = None  # release the previous solver first (outside the timed region)
        ms, (x, st, s) = event_ms(once)
        best = ms if best is None else min(best, ms)
    if cfg["type"] == "IterativeRefinement":  # the extended-precision solution
        x = s.phi(gb.FLOAT64)
    r = A.residual(x.double(), b, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
    rel = float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b.double()))
    return best, st, rel


def other_configs(gb, peak):
    """The reference's other benchmark configurations on the same GPU."""
    import numpy as np
    import torch
    out = {}
    # 32^3 Poisson, 64 tiles, PBiCGStab + ILU(0) to 1e-6.
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 32, 32, 32, 64)
    A = h.copyToTile()
    b = A * A.vector(gb.randomVector(0, h.numRows).astype(np.float32))
    ms, st, rel = timed_solve(gb, A, pbicgstab("ILU", 1e-6), b, reps=3)
    out["poisson32_pbicgstab_ilu0"] = {"ms": ms, "iterations": st.iterations, "converged": st.converged,
                                       "rel_residual_fp64": rel}
    # 128^3 upwind convection-diffusion (cell Peclet 0.5), 1024 tiles, to 1e-8,
    # Gauss-Seidel (2 sweeps) and ILU(0), FP32 and FP64.
    h = gb.generateMatrix(gb.GEN_CONVDIFF, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024)
    xt = gb.randomVector(1, h.numRows, "normal")
    for vt, name in [(gb.FLOAT32, "fp32"), (gb.FLOAT64, "fp64")]:
        hv = h if vt == gb.FLOAT32 else h.astype(gb.FLOAT64)
        A = hv.copyToTile()
        b = A * A.vector(xt.astype(np.float32 if vt == gb.FLOAT32 else np.float64))
        for pre in ("GS", "ILU"):
            ms, st, rel = timed_solve(gb, A, pbicgstab(pre, 1e-8, 2000), b)
            out[f"convdiff128_{pre.lower()}_{name}"] = {"ms": ms, "iterations": st.iterations,
                                                       "converged": st.converged, "rel_residual_fp64": rel}
        if vt == gb.FLOAT32:
            # One Gauss-Seidel sweep from a nonzero x (every entry read), back
            # to back on device; 8m + 20n algorithmic bytes (matrix values and
            # columns, row pointers, diagonal, b, x in, x out). The matrix
            # (133 MB) is larger than L2.
            gs1 = gb.Solver(A, {"type": "GaussSeidel", "numFixedIterations": 1})
            xg = A.vector(gb.randomVector(5, h.numRows).astype(np.float32))
            gs1.timeRepeated(xg, b, 3)
            ms = gs1.timeRepeated(xg, b, 20)
            byts = 8 * h.numOffDiag + 20 * h.numRows
            out["convdiff128_gs_sweep"] = {"ms": ms, "bytes_per_sweep": byts,
                                           "GBs": byts / (ms * 1e-3) / 1e9,
                                           "frac_of_hbm": byts / (ms * 1e-3) / 1e9 / peak,
                                           "kernel": "gsWarpRingKernel (one warp per tile)"}
            del gs1, xg
        del A
    # 100^3 LDU mesh (jittered, permuted), Gauss-Seidel PBiCGStab to 1e-8,
    # and the LDU SpMV (matrix smaller than L2: L2 flushed before each launch).
    # The matrix is nearly singular (diagonal = sum of face coefficients +
    # 1e-3): FP32 PBiCGStab reaches ~2e-8 and then diverges (the oracle does
    # the same), so FP32 runs a bounded number of iterations and reports the
    # residual it attains; FP64 and MPIR (FP32 inner solves) reach 1e-8.
    h = gb.generateLduMesh(100, 100, 100, 4, 5, 6, numTiles=1024)
    xt = gb.randomVector(1, h.numRows, "normal")
    A = h.copyToTile()
    b = A * A.vector(xt.astype(np.float32))
    ms, st, rel = timed_solve(gb, A, pbicgstab("GS", 1e-8, 260), b)
    out["ldu100_pbicgstab_gs_fp32_260it"] = {"ms": ms, "iterations": st.iterations, "converged": st.converged,
                                             "rel_residual_fp64": rel}
    gs_inner = {"type": "IterativeRefinement", "relResidual": 1e-8, "maxIterations": 20,
                "extendedPrecisionType": "float64", "innerSolver": pbicgstab("GS", 1e-4, 400)}
    ms, st, rel = timed_solve(gb, A, gs_inner, b)
    out["ldu100_mpir_gs"] = {"ms": ms, "outer": st.iterations, "inner": st.innerIterations,
                             "converged": st.converged, "rel_residual_fp64_of_phi": rel}
    A64 = h.astype(gb.FLOAT64).copyToTile()
    b64 = A64 * A64.vector(xt)
    ms, st, rel = timed_solve(gb, A64, pbicgstab("GS", 1e-8, 2000), b64)
    out["ldu100_pbicgstab_gs_fp64"] = {"ms": ms, "iterations": st.iterations, "converged": st.converged,
                                       "rel_residual_fp64": rel}
    del A64
    n, F = h.numRows, h.numOffDiag // 2
    y = torch.empty_like(b)
    t = A.timeSpmv(b, y, reps=20, flushL2=True)  # each launch alone between CUDA events, L2 flushed first
    ldu_bytes = 20 * n + 20 * F       # reference LDU arrays: cells 5 x 4 B, faces 5 x 4 B
    layout_bytes = 16 * F + 16 * n + 4  # this library's layout: 2F (col, value) pairs, diag, x, y, rowPtr
    out["ldu100_spmv"] = {"ms": t, "cells": n, "faces": F,
                          "GBs_ldu_algorithmic": ldu_bytes / (t * 1e-3) / 1e9,
                          "GBs_device_layout": layout_bytes / (t * 1e-3) / 1e9,
                          "frac_of_hbm_device_layout": layout_bytes / (t * 1e-3) / 1e9 / peak,
                          "l2": "flushed (256 MB write) before each launch"}
    return out


def serving(gb, requests=10000, slots=16, seed=7, rate_requests=2000, cold_requests=48, gen_threads=0,
            max_wall_s=300.0):
    """C5: a stream of solves, each a fresh 7-point variable-coefficient
    Poisson system (sigma 1) with grid edge L ~ U{16..96}, 70 % FP32
    PBiCGStab-ILU(0) to 1e-6 and 30 % MPIR to 1e-10 (by seed).

    Every request has its own coefficients (seed 100000 + k). Host threads
    generate the requests just ahead of their arrival: the values alone
    (gr_host_matrix_generate_values) on the layout of one template matrix
    per edge, submitted with gr_server_submit_values, so the client never
    holds more than a bounded number of systems. The server keeps one
    resident pair per (structure, configuration) and serves a request on a
    resident structure by uploading its values and refactorising in place.

    Saturation: all `requests` submitted as fast as they are generated;
    throughput = requests / (last finish - first arrival). Latency: Poisson
    arrivals at 50 %, 80 % and 100 % of that throughput, `rate_requests`
    each; p50 / p99 from arrival to result. Cold: `cold_requests` requests
    whose structures the server has never seen (tile layout, level rings,
    upload and factorisation all in the latency). A run that exceeds
    `max_wall_s` stops submitting and reports the requests it served
    ("truncated")."""
    import concurrent.futures as cf
    import numpy as np
    ilu = {"type": "PBiCGStab", "maxIterations": 1000, "relResidual": 1e-6, "preconditioner": {"type": "ILU"}}
    mpir = {"type": "IterativeRefinement", "relResidual": 1e-10, "maxIterations": 30,
            "extendedPrecisionType": "float64",
            "innerSolver": {"type": "PBiCGStab", "maxIterations": 500, "relResidual": 1e-4,
                            "preconditioner": {"type": "ILU"}}}
    rng = np.random.default_rng(seed)
    edges = rng.integers(16, 97, requests)
    kinds = rng.random(requests) < 0.3
    tiles = lambda L: max(1, (L ** 3 + 3455) // 3456)  # noqa: E731  (~3456 rows a tile)
    templates, tlock = {}, threading.Lock()

    def template(L):
        with tlock:
            if L not in templates:
                templates[L] = (threading.Lock(), None)
            lk, _ = templates[L]
        with lk:
            if templates[L][1] is None:
                templates[L] = (lk, gb.generateMatrix(gb.GEN_VAR_POISSON, L, L, L, (1.0,), 99, tiles(L)))
            return templates[L][1]

    def make(k, fresh_structure=False):
        L = int(edges[k % requests])
        cfg = mpir if kinds[k % requests] else ilu
        b = gb.randomVector(200000 + k, L ** 3).astype(np.float32)
        if fresh_structure:  # a structure nobody has seen: its own tile count
            return (gb.generateMatrix(gb.GEN_VAR_POISSON, L, L, L, (1.0,), 100000 + k, tiles(L) + 1 + k % 7),
                    None, b, cfg)
        tm = template(L)
        return tm, gb.generateValues(tm, gb.GEN_VAR_POISSON, L, L, L, (1.0,), 100000 + k), b, cfg

    threads = gen_threads or max(2, (os.cpu_count() or 4) - slots // 2)
    pool = cf.ThreadPoolExecutor(max_workers=threads)

    def run(srv, ks, rate, fresh_structure=False, ahead=256):
        """Submits requests ks (arrival times from `rate`, None: at once) and
        collects the results; generation runs `ahead` requests ahead."""
        gaps = rng.exponential(1.0 / rate, len(ks)) if rate else np.zeros(len(ks))
        futs, nxt = {}, 0

        def fill(i):
            nonlocal nxt
            while nxt < len(ks) and nxt < i + ahead:
                futs[nxt] = pool.submit(make, ks[nxt], fresh_structure)
                nxt += 1
        ids, pending = [], []
        lat, hits, conv = [], {0: 0, 1: 0, 2: 0}, True
        phases = {"queue": [], "setup": [], "solve": [], "device_solve": []}
        first_arrival, last_finish = None, None

        def collect(block):
            nonlocal conv, last_finish, first_arrival
            while pending and (block or len(pending) > 2 * slots + 64):
                rid = pending.pop(0)
                _, st, tm = srv.wait(rid)
                lat.append(tm["finished_ms"] - tm["arrival_ms"])
                phases["queue"].append(tm["admitted_ms"] - tm["arrival_ms"])
                phases["setup"].append(tm["solve_start_ms"] - tm["admitted_ms"])
                phases["solve"].append(tm["finished_ms"] - tm["solve_start_ms"])
                phases["device_solve"].append(st.solveMs)
                hits[tm["cache_hit"]] += 1
                conv = conv and st.converged
                first_arrival = tm["arrival_ms"] if first_arrival is None else min(first_arrival, tm["arrival_ms"])
                last_finish = tm["finished_ms"] if last_finish is None else max(last_finish, tm["finished_ms"])
        t0 = time.perf_counter()
        due = 0.0
        truncated = False
        for i in range(len(ks)):
            if time.perf_counter() - t0 > max_wall_s:
                truncated = True
                break
            fill(i)
            h, vals, b, cfg = futs.pop(i).result()
            due += gaps[i]
            d = due - (time.perf_counter() - t0)
            if rate and d > 0:
                time.sleep(d)
            pending.append(srv.submit(h, cfg, b) if vals is None else srv.submitValues(h, vals[0], vals[1], cfg, b))
            del h, vals, b
            collect(False)
        collect(True)
        for f in futs.values():
            f.cancel()
        lat = np.array(lat)
        span = (last_finish - first_arrival) * 1e-3
        return {"offered_per_s": rate, "requests": len(lat), "truncated": truncated,
                "throughput_per_s": len(lat) / span,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "all_converged": conv, "fresh_values_on_resident_structure": hits[2],
                "resident_same_matrix": hits[1], "new_pairs": hits[0],
                # Mean ms per request: waiting for a slot, values upload and
                # refactorisation, the solve with b in and x out, and the
                # solve's device time alone.
                "phases_mean_ms": {k: float(np.mean(v)) for k, v in phases.items()}}

    out = {"requests": requests, "slots": slots, "generator_threads": threads,
           "edges": "U{16..96}", "mix": "70 % FP32 PBiCGStab-ILU(0) 1e-6, 30 % MPIR 1e-10",
           "systems": "every request fresh coefficients (seed 100000 + k)"}
    srv = gb.Server(slots=slots)
    t0 = time.perf_counter()
    sat = run(srv, list(range(requests)), None)
    sat["wall_s"] = time.perf_counter() - t0
    res = {"saturation": sat}
    for f in ((0.5, 0.8, 1.0) if rate_requests > 0 else ()):
        ks = list(range(requests, requests + rate_requests))
        res[f"load_{f}"] = run(srv, ks, f * sat["throughput_per_s"])
    srv.close()
    out["stream"] = res
    if cold_requests > 0:
        srv = gb.Server(slots=slots)
        out["cold"] = run(srv, list(range(requests + rate_requests, requests + rate_requests + cold_requests)),
                          None, fresh_structure=True)
        srv.close()
    pool.shutdown()
    return out


def batching(gb, systems=64, seed=11, reps=3):
    """Many uneven systems: 7-point variable-coefficient Poisson (sigma 1),
    grid edge U{16..48}, FP32 PBiCGStab + ILU(0) (ring kernel) to 1e-6,
    host vectors in and out. One batch (gr_batch_solve_host: every launch
    covers all systems) against the same systems solved one after another
    by resident solvers (gr_solve_host); best of `reps` wall-clock passes,
    setup (upload, factorisation) excluded from both. The batch's solutions
    are compared bit for bit with the one-by-one ones."""
    import numpy as np
    rng = np.random.default_rng(seed)
    cfg = {"type": "PBiCGStab", "maxIterations": 1000, "relResidual": 1e-6,
           "preconditioner": {"type": "ILU", "kernel": "ring"}}
    hs, bs = [], []
    for k in range(systems):
        L = int(rng.integers(16, 49))
        hs.append(gb.generateMatrix(gb.GEN_VAR_POISSON, L, L, L, (1.0,), 3000 + k, max(1, L ** 3 // 3456)))
        bs.append(gb.randomVector(4000 + k, hs[-1].numRows).astype(np.float32))
    rows = sum(h.numRows for h in hs)
    solvers = [gb.Solver(h.copyToTile(), cfg) for h in hs]
    B = gb.Batch(hs, cfg)

    def one_by_one():
        xs, sts = [], []
        for s, h, b in zip(solvers, hs, bs):
            x = np.zeros(h.numRows, np.float32)
            sts.append(s.solveHost(x, b))
            xs.append(x)
        return xs, sts

    def best(fn):
        fn()
        t, out = None, None
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            dt = (time.perf_counter() - t0) * 1e3
            t = dt if t is None else min(t, dt)
        return t, out
    t_seq, (xs_seq, st_seq) = best(one_by_one)
    t_bat, (xs_bat, st_bat) = best(lambda: B.solveHost(bs))
    same = all(np.array_equal(a, b) for a, b in zip(xs_seq, xs_bat)) and \
        all(a.iterations == b.iterations for a, b in zip(st_seq, st_bat))
    its = [s.iterations for s in st_bat]
    B.close()
    return {"systems": systems, "rows_total": rows, "grid_edges": "U{16..48}",
            "iterations_min_max": [min(its), max(its)],
            "batch_ms": t_bat, "one_by_one_ms": t_seq,
            "batch_systems_per_s": systems / (t_bat * 1e-3),
            "one_by_one_systems_per_s": systems / (t_seq * 1e-3),
            "speedup": t_seq / t_bat, "identical_to_one_by_one": same,
            "all_converged": all(s.converged for s in st_bat)}


def _case_c1(gb):
    import numpy as np
    h = gb.generate3DPoissonMatrix(gb.FLOAT32, 32, 32, 32, 64)
    A = h.copyToTile()
    b = A * A.vector(gb.randomVector(0, h.numRows).astype(np.float32))
    return A, pbicgstab("ILU", 1e-6), b


def _case_c2(pre, vt_name):
    def build(gb):
        import numpy as np
        h = gb.generateMatrix(gb.GEN_CONVDIFF, 128, 128, 128, (0.5, 0.25, 0.125), 0, 1024)
        vt = gb.FLOAT32 if vt_name == "f32" else gb.FLOAT64
        hv = h if vt == gb.FLOAT32 else h.astype(gb.FLOAT64)
        A = hv.copyToTile()
        xt = gb.randomVector(1, h.numRows, "normal")
        b = A * A.vector(xt.astype(np.float32 if vt == gb.FLOAT32 else np.float64))
        return A, pbicgstab(pre, 1e-8, 2000), b
    return build


def _case_c3(kind):
    def build(gb):
        import numpy as np

        class _A:  # the bench's own defaults
            inner_maxit, inner_tol = 500, 1e-4
        h = gb.generateMatrix(gb.GEN_VAR_POISSON, 192, 192, 192, (1.5,), SEED_MATRIX, C3_TILES)
        xt = gb.randomVector(SEED_X, h.numRows).astype(np.float32)
        if kind == "fp64":
            A = h.astype(gb.FLOAT64).copyToTile()
            A32 = h.copyToTile()
            b = (A32 * A32.vector(xt)).double()
            del A32
            return A, FP64_CONFIG, b
        A = h.copyToTile()
        b = A * A.vector(xt)
        return A, mpir_config(_A, "twofloat32" if kind == "dw" else "float64"), b
    return build


def _case_c4(gb):
    import numpy as np
    h = gb.generateLduMesh(100, 100, 100, 4, 5, 6, numTiles=1024)
    A = h.copyToTile()
    b = A * A.vector(gb.randomVector(1, h.numRows, "normal").astype(np.float32))
    return A, pbicgstab("GS", 1e-8, 260), b


# One benchmark configuration each: (builder, description).
CASES = {
    "c1": (_case_c1, "32^3 Poisson, 64 tiles, FP32 PBiCGStab-ILU(0) to 1e-6"),
    "c2-gs-f32": (_case_c2("GS", "f32"), "128^3 convection-diffusion, 1024 tiles, FP32 PBiCGStab-GS(2) to 1e-8"),
    "c2-gs-f64": (_case_c2("GS", "f64"), "128^3 convection-diffusion, 1024 tiles, FP64 PBiCGStab-GS(2) to 1e-8"),
    "c2-ilu-f32": (_case_c2("ILU", "f32"), "128^3 convection-diffusion, 1024 tiles, FP32 PBiCGStab-ILU(0) to 1e-8"),
    "c2-ilu-f64": (_case_c2("ILU", "f64"), "128^3 convection-diffusion, 1024 tiles, FP64 PBiCGStab-ILU(0) to 1e-8"),
    "c3-mpir": (_case_c3("mpir"), f"192^3 var-coeff Poisson, {C3_TILES} tiles, MPIR FP64 outer / FP32 ILU inner"),
    "c3-mpir-dw": (_case_c3("dw"), f"192^3 var-coeff Poisson, {C3_TILES} tiles, MPIR double-word outer"),
    "c3-fp64": (_case_c3("fp64"), f"192^3 var-coeff Poisson, {C3_TILES} tiles, FP64 PBiCGStab-ILU(0) to 1e-10"),
    "c4-gs-f32": (_case_c4, "100^3 LDU mesh, 1024 tiles, FP32 PBiCGStab-GS(2), 260 iterations at most"),
    "c5": (None, "serving: 10,000 fresh variable-coefficient Poisson systems, edge U{16..96}, 70/30 ILU/MPIR"),
}


def run_case(a):
    """W untimed and K timed solves (solver creation + solve, CUDA events) of
    one configuration; one JSON line with the mean, iterations and the FP64
    relative residual of the last solution."""
    import torch
    import graphene_b200 as gb
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    build, desc = CASES[a.case]
    if build is None:  # serving
        t0 = time.perf_counter()
        res = serving(gb)
        print(json.dumps({"case": a.case, "workload": desc, "serving": res, "wall_s": time.perf_counter() - t0}))
        return 0
    A, cfg, b = build(gb)
    n = A.numRows

    def once():
        s = gb.Solver(A, cfg)
        x = torch.zeros(n, dtype=b.dtype, device="cuda")
        return s, x, s.solve(x, b)
    for _ in range(a.warmup):
        once()
    torch.cuda.synchronize()
    times, out = [], None
    l0 = gb.launch_count()
    for _ in range(a.steps):
        out = None
        ms, out = event_ms(once)
        times.append(ms)
    launches = gb.launch_count() - l0
    s, x, st = out
    xv = s.phi(gb.FLOAT64) if cfg["type"] == "IterativeRefinement" else x
    r = A.residual(xv, b, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
    rel = float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b.double()))
    print(json.dumps({"case": a.case, "workload": desc, "ms": statistics.mean(times) if times else None,
                      "ms_each": times, "iterations": st.iterations, "inner_iterations": st.innerIterations,
                      "converged": st.converged, "rel_residual_fp64": rel, "gpu_launches": launches,
                      "steps": a.steps, "warmup": a.warmup}))
    return 0


def event_ms(fn):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def main():
    a = parse_args()
    if a.impl == "reference":
        return reference_arm(a)
    if a.case:
        return run_case(a)
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
    peak, peak_kind = hbm_peak()
    clk = ClockSampler(torch.cuda.current_device()).start()

    t0 = time.perf_counter()
    h = gb.generateMatrix(gb.GEN_VAR_POISSON, a.grid, a.grid, a.grid, (a.sigma,), SEED_MATRIX, a.tiles)
    t_host = time.perf_counter() - t0
    n, m = h.numRows, h.numOffDiag
    A = h.copyToTile()
    xt = gb.randomVector(SEED_X, n).astype(np.float32)
    x_true = A.vector(xt)
    b = A * x_true  # b = A x in float32, as the reference's benchmark application does
    cfg = mpir_config(a)

    def solve(matrix, config, rhs):
        s = gb.Solver(matrix, config)
        x = torch.zeros(n, dtype=rhs.dtype, device="cuda")
        st = s.solve(x, rhs)
        return s, x, st

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(a.warmup):
        solve(A, cfg, b)
    barrier()
    clk.mark_start()
    launches0 = gb.launch_count()
    step_ms, stats = [], []
    s = x = None
    for _ in range(a.steps):
        # The previous step's solver is released before the next one is
        # built (outside the timed region), as a caller that rebuilds its
        # solver does; its device blocks are then reused.
        s = x = None
        ms, (s, x, st) = event_ms(lambda: solve(A, cfg, b))
        step_ms.append(ms)
        stats.append(st)
    barrier()
    launches = gb.launch_count() - launches0
    clk.mark_end()
    total = max_over_ranks(sum(step_ms), dist)
    ms_per_step = total / a.steps
    st = stats[-1]
    phi = s.phi(gb.FLOAT64)
    # Time-to-solution without solver creation (ILU factorisation, level-ring
    # packing, buffers): the last step's solver solves again from x0 = 0.
    resolve_ms = []
    for _ in range(max(3, a.steps)):
        xr = torch.zeros(n, dtype=torch.float32, device="cuda")
        ms_r, _ = event_ms(lambda: s.solve(xr, b))
        resolve_ms.append(ms_r)
    bnorm = float(torch.linalg.vector_norm(b.double()))

    def rel64(Amat, xv, rhs):
        r = Amat.residual(xv, rhs, destType=gb.FLOAT64, intermediateType=gb.FLOAT64)
        return float(torch.linalg.vector_norm(r)) / bnorm

    def best_of(fn, reps=2):
        """Fastest of `reps` runs (solver creation + solve, CUDA events) after
        one untimed run; the previous run's solver is released and collected
        before each timed run, so no teardown falls inside the timed region."""
        import gc
        out = fn()
        best = None
        for _ in range(reps):
            out = None
            gc.collect()
            torch.cuda.synchronize()
            ms, out = event_ms(fn)
            best = ms if best is None else min(best, ms)
        return best, out

    extra = {}
    # The extras (FP64 comparison, other configurations, serving, batching)
    # run in single-GPU runs only: replicas would repeat them on every rank
    # and contend for the host's cores.
    if not a.no_extras and world == 1:
        h64 = h.astype(gb.FLOAT64)
        A64 = h64.copyToTile()
        b64 = b.double()
        fp64_ms, (s64, x64, st64) = best_of(lambda: solve(A64, FP64_CONFIG, b64))
        extra["fp64_pbicgstab_ilu0"] = {"ms": fp64_ms, "iterations": st64.iterations,
                                        "converged": st64.converged,
                                        "rel_residual_fp64": rel64(A64, x64, b64)}
        extra["speedup_mpir_vs_fp64"] = fp64_ms / ms_per_step
        # The FP64 solve's kernels beside the FP32 ones below: where the
        # MPIR / FP64 ratio comes from (bytes: 12m + 28n for the SpMV, 12m +
        # 24n for the substitution's values, columns, inverse diagonal, b
        # in and x out).
        y64 = torch.empty_like(b64)
        A64.tuneSpmv(gb.FLOAT64, reps=5)
        spmv64_ms = A64.timeSpmv(b64, y64, reps=50, flushL2=False)  # each launch alone, matrix > L2
        ilu64 = gb.Solver(A64, {"type": "ILU"})
        z64 = torch.empty_like(b64)
        ilu64.timeRepeated(z64, b64, 3)
        ilu64_ms = ilu64.timeRepeated(z64, b64, 20)
        extra["fp64_kernels"] = {"spmv_ms": spmv64_ms, "spmv_GBs": (12 * m + 28 * n) / (spmv64_ms * 1e-3) / 1e9,
                                 "ilu0_apply_ms": ilu64_ms,
                                 "ilu0_apply_GBs": (12 * m + 24 * n) / (ilu64_ms * 1e-3) / 1e9,
                                 "per_iteration_ms": fp64_ms / max(1, st64.iterations)}
        del s64, x64, A64, h64, b64, y64, ilu64, z64
        for name, c in [("mpir_twofloat32", mpir_config(a, "twofloat32")),
                        ("mpir_float64_inner_tol_1e-3", mpir_config(a, "float64", 1e-3))]:
            ms, (sv, xv, sx) = best_of(lambda: solve(A, c, b))
            extra[name] = {"ms": ms, "outer": sx.iterations, "inner": sx.innerIterations,
                           "converged": sx.converged, "rel_residual_fp64": rel64(A, sv.phi(gb.FLOAT64), b)}
            del sv, xv
        extra["speedup_mpir_dw_vs_fp64"] = fp64_ms / extra["mpir_twofloat32"]["ms"]
        extra["configs"] = other_configs(gb, peak)
        extra["serving"] = serving(gb)
        extra["batching"] = batching(gb)

    # Kernel timings: SpMV and the ILU(0) application (HBM rooflines).
    y = torch.empty_like(x_true)
    tuned = A.tuneSpmv(gb.FLOAT32, reps=5)  # SpMV launch geometry (results unchanged)
    spmv_ms = A.timeSpmv(x_true, y, reps=50, flushL2=False)  # each launch alone, matrix > L2
    spmv_bytes = 8 * m + 16 * n + 4
    ilu = gb.Solver(A, {"type": "ILU"})
    z = torch.empty_like(x_true)
    ilu.timeRepeated(z, b, 3)
    ilu_ms = ilu.timeRepeated(z, b, 20)  # device time, launches back to back
    ilu_bytes = 8 * m + 12 * n
    gbs = lambda byts, ms: byts / (ms * 1e-3) / 1e9  # noqa: E731
    # Bytes the device layout itself moves: the 16-bit layout's 6-byte slots
    # and far columns (or 8-byte slots), chunk tables, diagonal, x and y.
    lay = A.spmvLayout()
    chunks = (n + 31) // 32
    lay_bytes = (lay["slots"] * (6 if lay["compact"] else 8) + 4 * lay["far"]
                 + 4 * (chunks + 1) * (2 if lay["compact"] else 1) + 12 * n)
    extra["spmv"] = {"ms": spmv_ms, "GBs": gbs(spmv_bytes, spmv_ms),
                     "frac_of_hbm": gbs(spmv_bytes, spmv_ms) / peak, "bytes_per_launch": spmv_bytes,
                     "layout": lay, "layout_bytes_per_launch": lay_bytes,
                     "layout_GBs": gbs(lay_bytes, spmv_ms), "layout_frac_of_hbm": gbs(lay_bytes, spmv_ms) / peak,
                     "autotuned_geometry": tuned}
    extra["ilu0_apply"] = {"ms": ilu_ms, "GBs": gbs(ilu_bytes, ilu_ms),
                           "frac_of_hbm": gbs(ilu_bytes, ilu_ms) / peak, "bytes_per_launch": ilu_bytes}
    if "fp64_kernels" in extra:
        extra["fp64_kernels"]["ilu0_apply_fp32_over_fp64"] = ilu_ms / extra["fp64_kernels"]["ilu0_apply_ms"]
        extra["fp64_kernels"]["spmv_fp32_over_fp64"] = spmv_ms / extra["fp64_kernels"]["spmv_ms"]
        st_inner = max(1, st.innerIterations)
        extra["fp64_kernels"]["mpir_per_inner_iteration_ms"] = ms_per_step / st_inner

    # End to end through the C ABI with pinned host buffers (natural order).
    b_host = torch.empty(n, dtype=torch.float32, pin_memory=True)
    b_host.copy_(torch.from_numpy(A.toNatural(b)))
    x_host = torch.zeros(n, dtype=torch.float32, pin_memory=True)
    e2e = []
    for i in range(min(a.steps, 3) + 1):
        x_host.zero_()
        ms, _ = event_ms(lambda: gb.Solver(A, cfg).solveHost(x_host.numpy(), b_host.numpy()))
        if i > 0:
            e2e.append(ms)
    err = float(np.abs(x_host.numpy() - xt).max())

    # Dominant kernel: two ILU(0) applications and two SpMVs per inner iteration.
    inner = st.innerIterations
    if 2 * inner * ilu_ms >= 2 * inner * spmv_ms:
        dom = ("ilu0_apply", "iluRingKernel", ilu_bytes, ilu_ms)
    else:
        dom = ("spmv", "spmvDotKernel", spmv_bytes, spmv_ms)
    # DRAM bytes per launch of the dominant kernel from the committed ncu
    # summary (a 160^3 capture of the two-tiles-a-block kernel the 192^3
    # solve runs, scaled by rows to one 192^3 launch).
    traffic = None
    tf = ROOT / "profiles" / "ilu_ring_grouped_var_poisson_160.md"
    if dom[0] == "ilu0_apply" and a.grid == 192 and tf.exists():
        import re
        hit = re.search(r"traffic_bytes_192: (\d+)", tf.read_text())
        traffic = int(hit.group(1)) if hit else None

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            threads = a.cpu_threads or os.cpu_count() or 1
            om, b_or = oracle_system(a, threads)
            smp = oracle_sample(om, b_or)
            tf_, ti_, tr_, ts_ = smp
            proj = project_ms(smp, st.iterations, inner)
            cpu = {"value": proj, "unit": "ms", "cores": threads, "kind": "port",
                   "sample": (f"oracle on the full {a.grid}^3 system ({threads} threads): ILU(0) "
                              f"factorisation {tf_:.2f} s, PBiCGStab-ILU(0) iterations {ti_:.3f} s each "
                              f"(solves of 1 and 4 iterations differenced), solve set-up {ts_:.3f} s, one "
                              f"FP64 residual {tr_:.3f} s, scaled to this solve's {inner} inner / "
                              f"{st.iterations} outer iterations")}
            if threads > 1:
                # The same sample on one thread (solves of 1 and 2 iterations).
                om.o.threads(1)
                smp1 = oracle_sample(om, b_or, k=1)
                cpu["single_thread"] = {"value": project_ms(smp1, st.iterations, inner),
                                        "unit": "ms", "cores": 1,
                                        "sample": (f"factorisation {smp1[0]:.2f} s, iterations {smp1[1]:.3f} s "
                                                   f"each (solves of 1 and 2 iterations differenced), one FP64 "
                                                   f"residual {smp1[2]:.3f} s, scaled the same way")}
        except Exception as e:
            cpu = {"value": None, "error": str(e)[:200]}
    clk.stop()

    line = {
        "metric": METRIC, "value": ms_per_step, "unit": "ms", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 outer",
        "data": "synthetic (seeded generator)",
        "config": bench_config(a, world),
        # The north-star comparison on the same GPU: plain FP64 PBiCGStab-ILU(0)
        # to 1e-10, and MPIR with a double-word outer residual.
        "fp64_ms": extra.get("fp64_pbicgstab_ilu0", {}).get("ms"),
        "speedup_mpir_vs_fp64": extra.get("speedup_mpir_vs_fp64"),
        "mpir_dw_ms": extra.get("mpir_twofloat32", {}).get("ms"),
        "speedup_mpir_dw_vs_fp64": extra.get("speedup_mpir_dw_vs_fp64"),
        "solve": {"outer_iterations": st.iterations, "inner_iterations": inner,
                  "converged": st.converged, "rel_residual_fp64_of_phi": rel64(A, phi, b),
                  "p50_ms": statistics.median(step_ms), "p99_ms": max(step_ms),
                  "step_ms": step_ms,
                  "p50_ms_excluding_setup": statistics.median(resolve_ms)},
        "extra": extra,
        "roofline": {"bound": "hbm", "kernel": dom[1], "achieved": gbs(dom[2], dom[3]),
                     "peak": peak, "unit": "GB/s", "frac": gbs(dom[2], dom[3]) / peak,
                     "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": dom[2], "launch_ms": dom[3]},
        "cpu_baseline": cpu,
        "e2e": {"value": statistics.mean(e2e), "unit": "ms", "h2d_bytes_per_step": 2 * 4 * n,
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


if __name__ == "__main__":
    sys.exit(main())
