#!/usr/bin/env python3
"""Benchmark of the steady SIMPLE hot path on one B200 (one process per GPU).

Workload (named by the benchmark's metric): the ~1M-tet straight pipe,
O-grid 24 rings x 72 sectors (+ an 18x18 square core) x 100 slabs, 6 tets per
quad and slab = 1,231,200 tets, seed-1 jitter of +-5 % local spacing, Re = 100,
alpha_u 0.7, alpha_p 0.3, pressure PCG rtol 1e-6 with the smoothed-aggregation
AMG + Chebyshev(2) V-cycle (the reference's plain path), FP64.

Metric: seconds to steady state (relCont <= 1e-6 and the pre-sweep momentum
audit <= 1e-6).  One full solve takes thousands of SIMPLE iterations, so a
benchmark "step" is one SIMPLE outer iteration of that solve (assembly,
momentum sweep, continuity, fine Schur refresh, AMG-PCG pressure solve,
pressure update) and

    value = STEADY_STATE_ITERATIONS x mean device seconds per step,

where STEADY_STATE_ITERATIONS is the iteration count of a complete solve of
this exact configuration by this solver (the CPU oracle follows the same
iteration history, see tests/), recorded in profiles/steady_state_pipe1m.md.
The per-iteration working set (fine CSR ~1 GB) is larger than the 126 MB L2.

Modes:
  python bench.py [--gpus N --steps K --warmup W]     this package (CUDA path)
  python bench.py --impl reference [...]                the CPU restatement of
      the reference's SIMPLE loop (oracle/, FP64, all host threads), same
      metric and workload, each step one SIMPLE iteration (bounded sample).
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

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "s to steady state (resid 1e-6): FP32+learned vs plain FP64 AMG-FGMRES, 1 B200"
WORKLOAD = "pipe1m"
OPTIONS = dict(re=100.0, alpha_u=0.7, alpha_p=0.3, p_rtol=1e-6, p_max=400, run_mode="converge", simple_tol=1e-6,
               max_outer=100000, amg_hierarchy="sa", amg_smoother="cheb2", pressure_solver="pcg")
# SIMPLE iterations of a complete solve of OPTIONS on WORKLOAD to relCont <= 1e-6
# plus the momentum audit (profiles/steady_state_pipe1m.md).
STEADY_STATE_ITERATIONS = {"fp64": 4193}
STEADY_STATE_SOURCE = "profiles/steady_state_pipe1m.md"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic():
    p = ROOT / "profiles" / "fine_spmv_traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("bytes_per_launch_pipe1m_fp64")
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _barrier_max(x: float, ws: int, device: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def fine_spmv_bytes(problem, s: int) -> float:
    """Compulsory bytes of one fine Schur SpMV: values + columns + row offsets + x + y."""
    row = problem.array("fine.row")
    n = len(row) - 1
    nnz = int(row[-1])
    return nnz * (s + 4) + 4 * (n + 1) + 2 * s * n


def sell_format_bytes(problem, s: int) -> float:
    """Bytes the SELL-32 fine operator actually streams per SpMV: padded
    values (s B) and 16-bit column deltas, slice offsets/widths, x and y."""
    row = problem.array("fine.row")
    n = len(row) - 1
    lens = np.diff(row)
    ns = (n + 31) // 32
    w = np.zeros(ns * 32, dtype=np.int64)
    w[:n] = lens
    padded = int(w.reshape(ns, 32).max(axis=1).sum()) * 32
    return padded * (s + 2) + 8 * ns + 2 * s * n


def run_nodals(args):
    from nodals_b200 import meshgen
    from nodals_b200 import native as N
    ws, rank, local = _dist()
    if ws > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    prec = args.precision
    tm = meshgen.named(WORKLOAD)
    mesh = N.Mesh.from_tetmesh(tm)
    t0 = time.perf_counter()
    P = N.Problem(mesh, precision=prec, device=local, **OPTIONS)
    setup_s = time.perf_counter() - t0
    S = N.Solver(P)
    for _ in range(args.warmup):
        S.step()
    l0 = N.launch_count()
    S.profile(True)
    _barrier_max(0.0, ws, local)
    with Clocks(local) as clk:
        dev_ms = []
        w0 = time.perf_counter()
        for _ in range(args.steps):
            r = S.step()
            dev_ms.append(r.ms_assembly + r.ms_momentum + r.ms_continuity + r.ms_pressure + r.ms_update)
        wall = time.perf_counter() - w0
    launches = N.launch_count() - l0
    prof = S.profile_read()
    S.profile(False)
    mean_ms = float(np.mean(dev_ms))
    mean_ms = _barrier_max(mean_ms, ws, local)
    n_ss = STEADY_STATE_ITERATIONS[prec] if WORKLOAD == "pipe1m" else 0
    value = n_ss * mean_ms / 1e3
    s_bytes = 8 if prec == "fp64" else 4
    calls, tot = prof["fine_spmv"]
    if calls == 0:
        raise RuntimeError("no fine SpMV launch was timed in the timed region")
    avg_launch_ms = tot / calls
    alg = fine_spmv_bytes(P, s_bytes)
    fmt = sell_format_bytes(P, s_bytes)
    peak, peak_kind = _peaks()
    achieved = alg / (avg_launch_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": _traffic(), "peak_kind": peak_kind,
            "kernel": "fine Schur SpMV of the PCG step (SELL-32, sell_spmv<double,3>)",
            "algorithmic_bytes_per_launch": int(alg),
            "algorithmic_bytes_rule": "nnz*(8+4) + 4(n+1) + 2*8*n (CSR index 4 B, value 8 B, x and y once)",
            "format_bytes_per_launch": int(fmt),
            "format_frac": round(fmt / (avg_launch_ms * 1e-3) / 1e9 / peak, 4),
            "avg_launch_ms": round(avg_launch_ms, 5), "launches": calls}

    # e2e: the public C ABI from host arrays: mesh -> setup -> device upload,
    # then per step H2D of the state (u, p) from pinned host memory, one SIMPLE
    # iteration, D2H of the new state.
    e2e = None
    if args.e2e:
        import torch
        torch.cuda.set_device(local)
        del S
        t0 = time.perf_counter()
        mesh2 = N.Mesh.from_tetmesh(tm)
        P2 = N.Problem(mesh2, precision=prec, device=local, **OPTIONS)
        S2 = N.Solver(P2)
        fixed_s = time.perf_counter() - t0
        c = P2.counts()
        hu = [torch.zeros(c["nv"], dtype=torch.float64).pin_memory() for _ in range(3)]
        hp = torch.zeros(c["nc"], dtype=torch.float64).pin_memory()
        ptrs = [x.data_ptr() for x in hu] + [hp.data_ptr()]
        import ctypes as C
        L = N.lib()

        def e2e_step():
            N._check(L.nds_set_fields(S2._h, *[C.c_void_p(p) for p in ptrs]))
            r = N.IterReport()
            N._check(L.nds_simple_step(S2._h, C.byref(r)))
            N._check(L.nds_get_fields(S2._h, *[C.c_void_p(p) for p in ptrs]))
        for _ in range(args.warmup):
            e2e_step()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        step_s = (time.perf_counter() - w0) / args.steps
        step_s = _barrier_max(step_s, ws, local)
        bytes_state = 8 * (3 * c["nv"] + c["nc"])
        e2e = {"value": round(fixed_s + n_ss * step_s, 3), "unit": "s", "h2d_bytes_per_step": bytes_state,
               "d2h_bytes_per_step": bytes_state, "fixed_setup_s": round(fixed_s, 3),
               "step_ms": round(step_s * 1e3, 4)}
        P = P2

    cpu = None
    if rank == 0 and ws == 1 and args.cpu_baseline:
        cpu = cpu_baseline(P, n_ss)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(mean_ms, 4), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32", "data": "synthetic (seeded pipe mesh)",
            "config": {"workload": f"{WORKLOAD}: straight pipe R=0.5 L=10, 1,231,200 tets (24x72 O-grid + 18x18 core, "
                                   f"100 slabs), Re=100, alpha_u=0.7, alpha_p=0.3, SA+cheb2 PCG rtol 1e-6",
                       "cells": int(P.counts()["nc"]), "velocity_dofs": int(P.counts()["nv"]),
                       "step": "one SIMPLE outer iteration of the steady-state solve",
                       "steady_state_iterations": n_ss, "steady_state_source": STEADY_STATE_SOURCE,
                       "l2": "working set per step > 126 MB L2 (fine CSR ~1 GB); no flush",
                       "parallelism": "replicas" if ws > 1 else "single GPU", "host_setup_s": round(setup_s, 3),
                       "wall_ms_per_step": round(wall / args.steps * 1e3, 4)},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(), "kernel_ms": {k: round(v[1], 3) for k, v in prof.items()},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(P, n_ss, max_seconds=25.0, max_steps=3):
    """The oracle (CPU FP64 restatement of the reference loop) on the host cores."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    O = Oracle(P, threads=threads)
    t0 = time.perf_counter()
    O.step()  # warm-up
    times = []
    while len(times) < max_steps and (time.perf_counter() - t0) < max_seconds:
        w = time.perf_counter()
        O.step()
        times.append(time.perf_counter() - w)
    t = float(np.mean(times))
    return {"value": round(n_ss * t, 3), "unit": "s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} SIMPLE iterations of the {WORKLOAD} steady-state solve after 1 warm-up "
                      f"({t:.3f} s each) x {n_ss} iterations"}


def run_reference(args):
    """CPU reference arm: oracle/h8_oracle.c on the same workload (rank 0 only)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from nodals_b200 import meshgen
    from nodals_b200 import native as N
    from oracle.oracle import Oracle
    P = N.Problem(N.Mesh.from_tetmesh(meshgen.named(WORKLOAD)), precision="fp64", **OPTIONS)
    threads = os.cpu_count() or 1
    O = Oracle(P, threads=threads)
    for _ in range(min(args.warmup, 1)):
        O.step()
    t0 = time.perf_counter()
    times = []
    while len(times) < args.steps and (time.perf_counter() - t0) < args.ref_seconds:
        w = time.perf_counter()
        O.step()
        times.append(time.perf_counter() - w)
    t = float(np.mean(times))
    n_ss = STEADY_STATE_ITERATIONS["fp64"]
    value = round(n_ss * t, 3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": ws,
            "steps": len(times), "warmup": min(args.warmup, 1), "ms_per_step": round(t * 1e3, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded pipe mesh)",
            "config": {"workload": f"{WORKLOAD} (as the CUDA arm)", "steady_state_iterations": n_ss,
                       "step": "one SIMPLE outer iteration (bounded sample)"},
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                             "sample": f"{len(times)} SIMPLE iterations x {n_ss}"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nodals", choices=["nodals", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64"])
    ap.add_argument("--workload", default=WORKLOAD, choices=["pipe1m", "pipe400k", "pipe40k"],
                    help="pipe1m is the benchmark; the smaller pipes serve kernel profiling only")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--ref-seconds", type=float, default=60.0)
    args = ap.parse_args()
    globals()["WORKLOAD"] = args.workload
    if args.warmup < 3 and args.impl == "nodals":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_nodals(args)


if __name__ == "__main__":
    main()
